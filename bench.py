#!/usr/bin/env python3
"""Throughput of the LCODE 3D xi step on B200: xi-steps/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision fp64|mixed|fft32] [--grid 641]

Workload (default): the production grid of the reference's example config,
641 x 641 cells, h = 0.025 (window +-8), plasma coarseness 3 / fineness 2
(42,025 coarse and 1,537,600 fine particles), xi_step = 0.005, cold uniform
plasma, axisymmetric beam rho_b = A exp(-r^2/2) 0.5 (1 - cos(sqrt(pi/2) xi))
with A = 0.5 (blowout regime). Synthetic inputs: the plasma and beam are
generated, there is no dataset. The state is first advanced (untimed) into
the beam so the timed steps see the nonlinear wake.

One "step" is one full xi step (estimate, predictor, corrector, final move +
deposit: 3 pushes, 3 depositions, 2 field solves of 6 fields).

value: device-resident inputs (beam arrays already in HBM), context-owned
state, each step timed with CUDA events on the launching stream; L2 is
flushed (a 256 MiB write) between timed steps, outside the timed events.
stages_ms_per_step and the roofline's kernel time come from K further steps
with every kernel launch bracketed by CUDA events (kept out of `value`).
e2e: the same metric through the public drop-in API (lcode3d_b200.step) with
the beam copied host->device from pinned memory and Ez(0,0) read back
device->host every step, like the reference's CLI loop.

--impl reference: the reference algorithm on the host cores (the oracle
restatement in oracle/: numpy + scipy.fft, its particle kernels in C with
OpenMP), a bounded number of steps of the same workload.

Multi-GPU (torchrun, one process per GPU): a single simulation does not
shard (each step has global spectral solves), so every rank runs an
independent replica; value = all ranks' steps / max-over-ranks time.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = 'xi-steps/s'
GRIDS = {
    # N: (h, dxi, amplitude)
    641: (0.025, 0.005, 0.5),
    161: (0.05, 0.05, 0.05),
}


def make_config(N, precision):
    import types
    h, dxi, A = GRIDS[N]
    c = types.SimpleNamespace(
        grid_steps=N, grid_step_size=h, xi_step_size=dxi, xi_steps=3000,
        diagnostics_each_N_steps=10 ** 9, field_solver_subtraction_trick=1,
        field_solver_variant_A=True, reflect_padding_steps=5, plasma_padding_steps=10,
        plasma_coarseness=3, plasma_fineness=2, gpu_index=0, lc3d_precision=precision)

    def beam(xi_i, x, y):
        xi = xi_i * dxi
        if xi < 0 or xi > 2 * np.sqrt(2 * np.pi):
            return 0
        return A * np.exp(-(x ** 2 + y ** 2) / 2) * 0.5 * (1 - np.cos(np.sqrt(np.pi / 2) * xi))
    c.beam = beam
    return c


def beam_np(cfg, xi_i, xs, ys):
    N = cfg.grid_steps
    return np.broadcast_to(np.asarray(cfg.beam(xi_i, xs, ys), dtype=np.float64), (N, N)).copy()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------

class Clocks:
    Q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
         'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
         'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ['nvidia-smi', f'--id={self.index}', f'--query-gpu={self.Q}',
                 '--format=csv,noheader,nounits', '-lms', '100'],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, ValueError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['nvidia-smi unavailable']}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ('hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap')
        for ln in self.lines:
            f = [x.strip() for x in ln.split(',')]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith('active'):
                    reasons.add(n)
        return {'sm_mhz': statistics.median(sm) if sm else None, 'sm_max_mhz': mx,
                'reasons': sorted(reasons), 'samples': len(sm)}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def peaks():
    p = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get('hbm_gbs', 6650.0), 'measured (MEASURED_PEAKS.json)'
    return 6650.0, 'fallback (6.65 TB/s)'


def tensor_peak():
    p = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get('bf16_tflops', 1590.0), 'measured bf16 burst (MEASURED_PEAKS.json)'
    return 1590.0, 'fallback bf16 burst (1.59 PFLOP/s)'


def fp64_peak_tflops(torch):
    """FP64 denominator measured in this run: cuBLAS DGEMM 8192^3 (best of
    5), since the measured-peaks file holds no float64 figure."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device='cuda')
    b = torch.randn(n, n, dtype=torch.float64, device='cuda')
    torch.matmul(a, b)
    best = 1e9
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 2 * n ** 3 / (best * 1e-3) / 1e12


def tf32_peak_tflops(torch):
    """TF32 denominator measured in this run: cuBLAS float32 GEMM 8192^3 with
    TF32 tensor cores allowed (best of 5); the measured-peaks file holds
    no TF32 figure."""
    n = 8192
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = True
    a = torch.randn(n, n, dtype=torch.float32, device='cuda')
    b = torch.randn(n, n, dtype=torch.float32, device='cuda')
    torch.matmul(a, b)
    best = 1e9
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    torch.backends.cuda.matmul.allow_tf32 = prev
    del a, b
    torch.cuda.empty_cache()
    return 2 * n ** 3 / (best * 1e-3) / 1e12


def transform_flops_per_launch(N):
    """Algorithmic flops of one batched transform-GEMM launch: the 4 launches
    of a solve apply L and R to each of the 6 fields (r x c with r, c in
    {N, N-2}); each field costs 4 r c (r + c) flops over the 4 launches."""
    M = N - 2
    dims = [(N, M), (M, N), (M, M), (M, N), (N, M), (N, N)]
    return sum(4 * r * c * (r + c) for r, c in dims) / 4


def fft_bytes_per_launch(N, fp32=False):
    """Algorithmic bytes of one FFT row pass over the 6 fields of a solve,
    averaged over the 4 passes: every field's r x c array is read once and
    written once per pass, and one pass also reads the eigenvalue matrix.
    float64: 8 bytes per element everywhere (8 + 8, plus 8 / 4 for the
    eigenvalues). float32 transforms: the first pass reads float64 and
    writes float32, the last reads float32 and writes float64, the
    intermediates and eigenvalues are float32 (44 bytes per element over
    the 4 passes)."""
    M = N - 2
    dims = [(N, M), (M, N), (M, M), (M, N), (N, M), (N, N)]
    per = 44 / 4 if fp32 else 8 * (2 + 0.25)
    return sum(per * r * c for r, c in dims)


def deposit_bytes_per_launch(N, Nc, Nf):
    """Algorithmic bytes of one deposition (kernel + finalize): read the 7
    coarse arrays and the 5 fine-lattice arrays, read ro_initial, write
    ro, jx, jy, jz."""
    return 8 * (7 * Nc * Nc + 5 * Nf + N * N + 4 * N * N)


def run_ours(args, rank, world, dist):
    import torch
    import lcode3d_b200 as L
    from lcode3d_b200 import _lib

    dev = int(os.environ.get('LOCAL_RANK', 0))
    torch.cuda.set_device(dev)
    cfg = make_config(args.grid, args.precision)
    cfg.lc3d_fp64_transform = args.fp64_transform
    cfg.lc3d_mixed_slices = args.slices
    N = cfg.grid_steps
    xs, ys, const, virt, st = L.init(cfg)
    # the e2e loop's beams in pinned host memory, allocated first: pinning
    # memory has side effects on the host that slow the steps that follow it
    # for a while, which must not fall into a timed region
    K, W = args.steps, args.warmup
    pinned = [torch.from_numpy(beam_np(cfg, args.pre + i, xs, ys)).pin_memory() for i in range(W + K)]
    s = L.solver_for(cfg)
    s.set_virt(virt)
    s.set_const(const)
    L.lcode.check_errors = False
    stream = torch.cuda.current_stream()
    sp = ctypes.c_void_p(stream.cuda_stream)

    # advance (untimed) into the beam with the public API
    t_pre = time.time()
    ez_pre = []   # reduced precisions: Ez(N/2, N/2) of the pre-steps, for the float64 comparison
    for i in range(args.pre):
        st = L.step(cfg, const, virt, st, beam_np(cfg, i, xs, ys))
        if args.precision != 'fp64':
            ez_pre.append(st.Ez[N // 2, N // 2].clone())
    ez_field_pre = st.Ez.clone() if args.precision != 'fp64' and args.pre else None
    torch.cuda.synchronize()
    t_pre = time.time() - t_pre
    x0 = args.pre
    lib = _lib.lib
    names = _lib.STATE_NAMES
    ptrs = _lib.StatePtrs(*[getattr(st, n).data_ptr() for n in names])
    _lib.check(lib.lc3d_set_state(s.ctx, ctypes.byref(ptrs), sp), 'set_state')
    beams = [torch.from_numpy(beam_np(cfg, x0 + i, xs, ys)).cuda() for i in range(W + 2 * K)]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device='cuda')
    for i in range(W):
        _lib.check(lib.lc3d_step(s.ctx, ctypes.c_void_p(beams[i].data_ptr()), sp), 'step')
    torch.cuda.synchronize()
    _lib.check(lib.lc3d_check_error(s.ctx, sp), 'warmup')
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    _lib.check(lib.lc3d_profile(s.ctx, 0), 'profile reset')   # count launches, no per-launch events
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(dev)
    clocks.start()
    for i in range(K):
        flush.fill_(float(i))
        ev[i][0].record(stream)
        _lib.check(lib.lc3d_step(s.ctx, ctypes.c_void_p(beams[W + i].data_ptr()), sp), 'step')
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    ms_steps = [a.elapsed_time(b) for a, b in ev]
    nst = len(_lib.STAGES)
    launches = (ctypes.c_longlong * nst)()
    lib.lc3d_profile_read(s.ctx, launches, None, None)
    _lib.check(lib.lc3d_check_error(s.ctx, sp), 'timed steps')

    # ---- stage breakdown: K further steps, every launch bracketed by CUDA events ----
    _lib.check(lib.lc3d_profile(s.ctx, 1), 'profile')
    for i in range(K):
        flush.fill_(float(i))
        _lib.check(lib.lc3d_step(s.ctx, ctypes.c_void_p(beams[W + K + i].data_ptr()), sp), 'step')
    plaunches = (ctypes.c_longlong * nst)()
    kms = (ctypes.c_double * nst)()
    timed = (ctypes.c_longlong * nst)()
    lib.lc3d_profile_read(s.ctx, plaunches, kms, timed)
    lib.lc3d_profile(s.ctx, 0)
    _lib.check(lib.lc3d_check_error(s.ctx, sp), 'profiled steps')
    total_ms = sum(ms_steps)
    if dist:
        t = torch.tensor([total_ms], dtype=torch.float64, device='cuda')
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t)
    value = world * K / (total_ms * 1e-3)
    stage = {n: {'launches': int(plaunches[k]), 'ms': kms[k], 'timed': int(timed[k])}
             for k, n in enumerate(_lib.STAGES)}

    # ---- e2e through the public API, host beam in pinned memory ----
    st_e = st
    L.lcode.check_errors = True   # the drop-in default: the device error flag is read after every call
    for i in range(W):
        st_e = L.step(cfg, const, virt, st_e, pinned[i])
        float(st_e.Ez[N // 2, N // 2])
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record(stream)
    wall = []
    for i in range(K):
        ta = time.perf_counter()
        st_e = L.step(cfg, const, virt, st_e, pinned[W + i])
        float(st_e.Ez[N // 2, N // 2])   # D2H of the step's result
        wall.append((time.perf_counter() - ta) * 1e3)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    wall_ms = (time.perf_counter() - t0) * 1e3
    if dist:
        t = torch.tensor([e2e_ms], dtype=torch.float64, device='cuda')
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t)
    L.lcode.check_errors = True
    s.check_device_flag('e2e')

    # ---- the same steps as CUDA-graph replays (lc3d_run, device beam) ----
    bp = _lib.BeamParams(GRIDS[args.grid][2], 1.0, 1.0)
    _lib.check(lib.lc3d_set_beam(s.ctx, ctypes.byref(bp)), 'set_beam')
    ezh = torch.empty(W + K, dtype=torch.float64, device='cuda')
    xg = x0 + W + 2 * K   # the context state has advanced by W + 2K steps
    _lib.check(lib.lc3d_run(s.ctx, xg, W, ctypes.c_void_p(ezh.data_ptr()), sp), 'graph warmup')
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record(stream)
    _lib.check(lib.lc3d_run(s.ctx, xg + W, K, ctypes.c_void_p(ezh.data_ptr()), sp), 'graph run')
    g1.record(stream)
    torch.cuda.synchronize()
    graph_ms = g0.elapsed_time(g1)
    if dist:
        t = torch.tensor([graph_ms], dtype=torch.float64, device='cuda')
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        graph_ms = float(t)
    _lib.check(lib.lc3d_check_error(s.ctx, sp), 'graph run')

    if rank != 0:
        return None
    # ---- roofline of the dominant kernel ----
    dom = max(stage, key=lambda n: stage[n]['ms'])
    hbm, hbm_src = peaks()
    roof = None
    use_fft = args.fp64_transform != 'dense'
    if dom == 'transform' and stage[dom]['timed'] and args.precision in ('mixed', 'tf32'):
        avg_ms = stage[dom]['ms'] / stage[dom]['timed']
        S = args.slices or (4 if args.precision == 'mixed' else 3)
        fl = transform_flops_per_launch(N) * S * (S + 1) / 2
        ach = fl / (avg_ms * 1e-3) / 1e12
        if args.precision == 'tf32':
            pk, src = tf32_peak_tflops(torch), 'measured in this run: cuBLAS TF32 GEMM 8192^3 (no TF32 figure on file)'
        else:
            pk, src = tensor_peak()
        kname = 'BF16' if args.precision == 'mixed' else 'TF32'
        roof = {'kernel': f'oz_gemm_kernel (tcgen05 split-{kname} transforms, {S} slices, {S * (S + 1) // 2} products)',
                'bound': 'tensor', 'achieved': ach, 'peak': pk, 'unit': 'TFLOP/s', 'frac': ach / pk,
                'peak_source': src, 'algorithmic_per_launch': fl, 'avg_launch_ms': avg_ms, 'traffic': None}
    elif dom == 'transform' and stage[dom]['timed'] and (use_fft or args.precision == 'fft32'):
        avg_ms = stage[dom]['ms'] / stage[dom]['timed']
        f32 = args.precision == 'fft32'
        by = fft_bytes_per_launch(N, f32)
        ach = by / (avg_ms * 1e-3) / 1e9
        roof = {'kernel': f'fft_rows_kernel ({"FP32" if f32 else "FP64"} DST/DCT row-FFT pass, 6 fields)',
                'bound': 'hbm',
                'achieved': ach, 'peak': hbm, 'unit': 'GB/s', 'frac': ach / hbm,
                'peak_source': hbm_src, 'algorithmic_per_launch': by, 'avg_launch_ms': avg_ms,
                'traffic': None,
                'note': ('the rows stay in L2 (ncu: L2 throughput ~0.14 of peak); while active the pass is '
                         'bound by the L1/shared-memory pipe (~0.72 of peak) and by its barrier-separated radix '
                         'passes: profiles/fft_rows_kernel_641.md')}
    elif dom == 'transform' and stage[dom]['timed']:
        avg_ms = stage[dom]['ms'] / stage[dom]['timed']
        fl = transform_flops_per_launch(N)
        ach = fl / (avg_ms * 1e-3) / 1e12
        pk = fp64_peak_tflops(torch)
        roof = {'kernel': 'dgemm_kernel (FP64 DST/DCT transforms)', 'bound': 'fp64',
                'achieved': ach, 'peak': pk, 'unit': 'TFLOP/s', 'frac': ach / pk,
                'peak_source': 'measured in this run: cuBLAS DGEMM 8192^3 (MEASURED_PEAKS.json has no FP64 figure)',
                'algorithmic_per_launch': fl, 'avg_launch_ms': avg_ms, 'traffic': None}
    else:
        avg_ms = stage[dom]['ms'] / max(1, stage[dom]['timed'])
        by = deposit_bytes_per_launch(N, s.Nc, s.Nf)
        ach = by / (avg_ms * 1e-3) / 1e9
        roof = {'kernel': dom, 'bound': 'hbm', 'achieved': ach, 'peak': hbm, 'unit': 'GB/s',
                'frac': ach / hbm, 'peak_source': hbm_src, 'algorithmic_per_launch': by,
                'avg_launch_ms': avg_ms, 'traffic': None}
    tr = os.path.join(ROOT, 'profiles', 'traffic.json')
    if os.path.exists(tr):
        with open(tr) as f:
            t = json.load(f).get(f'{args.grid}_{args.precision}', {})
        if roof['kernel'].split(' ')[0] in t:
            roof['traffic'] = t[roof['kernel'].split(' ')[0]]
    out = {
        'metric': METRIC, 'value': value, 'unit': 'xi-steps/s', 'n_gpus': world,
        'steps': K, 'warmup': W, 'ms_per_step': total_ms / K, 'higher_is_better': True,
        'scaling': 'weak', 'vs_baseline': None,
        'dtype': {'fp64': 'f64', 'mixed': 'f64+bf16', 'fft32': 'f64+f32', 'tf32': 'f64+tf32'}[args.precision],
        'data': 'synthetic (generated cold uniform plasma + axisymmetric beam; no dataset)',
        'config': {'workload': f'LCODE 3D xi step, {N}x{N} grid, h={cfg.grid_step_size}, '
                               f'xi_step={cfg.xi_step_size}, coarseness 3 / fineness 2, A={GRIDS[N][2]}, '
                               f'{args.precision} field solvers',
                   'grid_steps': N, 'coarse_particles': s.Nc ** 2, 'fine_particles': s.Nf ** 2,
                   'precision': args.precision, 'fp64_transform': args.fp64_transform,
                   'mixed_slices': (args.slices or (4 if args.precision == 'mixed' else 3))
                   if args.precision in ('mixed', 'tf32') else None,
                   'start_xi_step': x0,
                   'l2': 'flushed between timed steps (256 MiB write, outside the step events)',
                   'parallelism': f'replicas x{world}' if world > 1 else 'single GPU'},
        'e2e': {'value': world * K / (e2e_ms * 1e-3), 'unit': 'xi-steps/s',
                'h2d_bytes_per_step': N * N * 8, 'd2h_bytes_per_step': 8 + 4,
                'error_check': 'device error flag read after every step (lcode.check_errors = True, the default)',
                'wall_ms': wall_ms, 'api': 'lcode3d_b200.step (drop-in for lcode.step)',
                'step_wall_ms': {'min': min(wall), 'median': statistics.median(wall), 'max': max(wall)}},
        'gpu_launches': int(sum(launches)),
        'launches_per_step': sum(launches) / K,
        'stages_ms_per_step': {n: stage[n]['ms'] / K for n in stage},
        'roofline': roof,
        'clocks': clk,
        'pre_steps_seconds': t_pre,
        'graph': {'value': world * K / (graph_ms * 1e-3), 'ms_per_step': graph_ms / K,
                  'how': 'the same K steps as one lc3d_run: CUDA-graph replay per step, beam evaluated '
                         'on the device, Ez(0,0) recorded on the device, no L2 flush between steps'},
    }
    if ez_field_pre is not None:
        out['accuracy_vs_fp64'] = accuracy_vs_fp64(args, ez_pre, ez_field_pre)
    return out


def accuracy_vs_fp64(args, ez_pre, ez_field_pre):
    """Ez of the reduced-precision pre-steps against the same steps in
    float64 from the same initial state: the on-axis Ez(N/2, N/2) history
    and the final Ez field, each as max |difference| / max |float64|."""
    import torch
    import lcode3d_b200 as L
    cfg = make_config(args.grid, 'fp64')
    N = cfg.grid_steps
    xs, ys, const, virt, st = L.init(cfg)
    ez = []
    for i in range(args.pre):
        st = L.step(cfg, const, virt, st, beam_np(cfg, i, xs, ys))
        ez.append(st.Ez[N // 2, N // 2].clone())
    h64 = torch.stack(ez).cpu().numpy()
    h = torch.stack(ez_pre).cpu().numpy()
    f64 = st.Ez.cpu().numpy()
    f = ez_field_pre.cpu().numpy()
    e_h = float(np.abs(h - h64).max() / max(np.abs(h64).max(), 1e-300))
    e_f = float(np.abs(f - f64).max() / max(np.abs(f64).max(), 1e-300))
    return {'steps': args.pre, 'ez_axis_history_max_rel': e_h, 'ez_field_max_rel': e_f,
            'within_1e-6': bool(max(e_h, e_f) <= 1e-6)}


ACCURACY_FIELDS = ('Ex', 'Ey', 'Ez', 'Bx', 'By', 'Bz', 'ro', 'jx', 'jy', 'jz')


def run_accuracy_table(args):
    """Error of every reduced-precision form against the float64 path on the
    641^2 production run (A = 0.5, dxi = 0.005) from its initial state: the
    max |difference| / max |float64| of each field at the given steps, and of
    the on-axis Ez(N/2, N/2) history up to each of them. Host beams through
    the drop-in step(), as the reference's loop evaluates them."""
    import torch
    import lcode3d_b200 as L
    torch.cuda.set_device(int(os.environ.get('LOCAL_RANK', 0)))
    N = args.grid
    marks = sorted(int(x) for x in args.accuracy_steps.split(','))
    steps = marks[-1]
    forms = [('fp64', {})] + [(f, {}) for f in ('fft32',) if f in args.forms.split(',')]
    forms += [(f'mixed_s{S}', {'lc3d_mixed_slices': S}) for S in (3, 4, 5)
              if f'mixed_s{S}' in args.forms.split(',')]
    forms += [(f'tf32_s{S}', {'lc3d_mixed_slices': S}) for S in (2, 3)
              if f'tf32_s{S}' in args.forms.split(',')]
    beams = None
    results, ref = {}, None
    for name, extra in forms:
        prec = name.split('_')[0]
        cfg = make_config(N, prec)
        for k, v in extra.items():
            setattr(cfg, k, v)
        xs, ys, const, virt, st = L.init(cfg)
        if beams is None:
            beams = [torch.from_numpy(beam_np(cfg, i, xs, ys)) for i in range(steps)]
        ez, snaps = [], {}
        t0 = time.perf_counter()
        for i in range(steps):
            st = L.step(cfg, const, virt, st, beams[i])
            ez.append(st.Ez[N // 2, N // 2].clone())
            if i + 1 in marks:
                snaps[i + 1] = {f: getattr(st, f).clone() for f in ACCURACY_FIELDS}
        torch.cuda.synchronize()
        secs = time.perf_counter() - t0
        hist = torch.stack(ez)
        if ref is None:
            ref = (hist, snaps)
            results[name] = {'seconds': secs}
            continue
        rows = {}
        for m in marks:
            r = {f: float((snaps[m][f] - ref[1][m][f]).abs().max() / ref[1][m][f].abs().max().clamp_min(1e-300))
                 for f in ACCURACY_FIELDS}
            h = (hist[:m] - ref[0][:m]).abs().max() / ref[0][:m].abs().max().clamp_min(1e-300)
            r['Ez_axis_history'] = float(h)
            rows[str(m)] = r
        e_h = rows[str(steps)]['Ez_axis_history']
        results[name] = {'seconds': secs, 'errors_vs_fp64': rows,
                         'ez_gate_1e-6': bool(e_h <= 1e-6 and rows[str(steps)]['Ez'] <= 1e-6)}
        del snaps
    return {'accuracy_table': results, 'grid_steps': N, 'steps': steps, 'marks': marks,
            'workload': f'{N}^2 production run, h={GRIDS[N][0]}, xi_step={GRIDS[N][1]}, A={GRIDS[N][2]}, '
                        'from the initial state, host beams through lcode3d_b200.step',
            'metric': 'max |form - fp64| / max |fp64| per field at each step; Ez(N/2, N/2) history up to it'}


# ---------------------------------------------------------------------------
# CPU: the oracle (reference algorithm) on the host cores
# ---------------------------------------------------------------------------

def time_oracle(grid, steps, threads, start, warmup=0):
    """xi-steps/s of the oracle over `steps` steps that begin at xi step
    `start` (the state is first advanced there, untimed), after `warmup`
    untimed steps. The beam arrays are evaluated before the timed loop, as
    the GPU arms have theirs ready before their timed regions."""
    from oracle import lcode_oracle as O
    O.use_c_kernels(threads)
    O.FFT_WORKERS = threads
    cfg = make_config(grid, 'fp64')
    xs, ys, const, virt, st = O.init(cfg)
    for i in range(start + warmup):
        st = O.step(cfg, const, virt, st, beam_np(cfg, i, xs, ys))
    x0 = start + warmup
    beams = [beam_np(cfg, x0 + i, xs, ys) for i in range(steps)]
    t0 = time.perf_counter()
    for i in range(steps):
        st = O.step(cfg, const, virt, st, beams[i])
    return steps / (time.perf_counter() - t0)


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_scan(args, rank, world, dist):
    """Batched parameter scan: args.scan simulations drawn (seeded) over the
    grids 161/321/481/641 with the window kept at +-8, dxi = 0.01, beam
    amplitude log-uniform [0.01, 1], sigma_r U[0.5, 2], length factor
    U[0.5, 1.5]; partitioned over ranks by cost, each rank's share advanced
    with one CUDA-graph launch per xi step. value = all simulations' steps /
    the slowest rank's time."""
    import torch
    from lcode3d_b200 import batch as B

    torch.cuda.set_device(int(os.environ.get('LOCAL_RANK', 0)))
    specs = B.scan_specs(args.scan, args.seed)
    mine = B.partition(specs, world)[rank]
    grids = sorted({specs[i]['grid_steps'] for i in mine})
    choice, timings = B.autotune(grids, steps=4)
    torch.cuda.synchronize()
    t_setup = time.perf_counter()
    multi = args.scan_deposit == 'multi'
    bt = B.Batch([specs[i] for i in mine], transform={N: c['transform'] for N, c in choice.items()},
                 tiles={N: (c['deposit_rows'], c['fft_ctas_per_sm']) for N, c in choice.items()},
                 multi_deposit=multi)
    torch.cuda.synchronize()
    t_setup = time.perf_counter() - t_setup
    K, W = args.steps, args.warmup
    bt.run(W)
    from lcode3d_b200 import _lib

    def read_launches():   # kernel launches counted by every context since the last read
        n = len(_lib.STAGES)
        tot = 0
        for sim in bt.sims:
            arr = (ctypes.c_longlong * n)()
            _lib.lib.lc3d_profile_read(sim.solver.ctx, arr, None, None)
            tot += sum(arr)
        return tot
    read_launches()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = Clocks(int(os.environ.get('LOCAL_RANK', 0)))
    clocks.start()
    e0.record(stream)
    hist = bt.run(K)
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = read_launches()
    bt.check_errors()
    ms = B.max_over_ranks(e0.elapsed_time(e1), dist)
    last = B.gather_histories({i: h[-1:].cpu().numpy() for i, h in zip(mine, hist)}, dist)
    if rank != 0:
        return None
    counts = {N: sum(1 for s in specs if s['grid_steps'] == N) for N in B.GRIDS}
    return {
        'metric': 'aggregate xi-steps/s (batched scan)', 'value': len(specs) * K / (ms * 1e-3),
        'unit': 'xi-steps/s', 'n_gpus': world, 'steps': K, 'warmup': W, 'ms_per_step': ms / K,
        'higher_is_better': True, 'scaling': 'strong', 'vs_baseline': None, 'dtype': 'f64',
        'data': 'synthetic (seeded scan draws, generated plasma and beams)',
        'config': {'workload': f'{len(specs)} independent simulations, grids {counts}, window +-8, dxi 0.01',
                   'seed': args.seed, 'l2': 'no flush (each batch step touches several GB, far more than L2)',
                   'deposition': ('one launch over all simulations per deposition point (4-row tiles)' if multi
                                  else 'per simulation, on its graph branch (autotuned tile rows)')},
        'autotune': {'choice': {str(k): v for k, v in choice.items()},
                     'ms_per_step': {str(k): v for k, v in timings.items()}},
        'gpu_launches': launches,
        'launches_per_batch_step': launches / K,
        'setup_s': t_setup,
        'all_final_Ez00_finite': bool(all(np.isfinite(v).all() for v in last.values())),
        'clocks': clk,
    }


def run_learned_bench(args):
    """The learned first pass on the bench workload: ``pre`` plain steps into
    the beam, W warm-up and K timed steps under periodic verification
    (lcode3d_b200.predictor.learned_steps; verification syncs included in
    the timed region), and the same K steps by the plain method from the
    same state for the Ez(N/2, N/2) error and the same-GPU comparison."""
    import torch
    from lcode3d_b200 import predictor as P
    from lcode3d_b200 import train_predictor as T

    dev = int(os.environ.get('LOCAL_RANK', 0))
    torch.cuda.set_device(dev)
    path = T.DEFAULT_WEIGHTS if args.learned == 'default' else args.learned
    if not os.path.exists(path):
        return {'impl': 'ours', 'form': 'fp64+learned',
                'unavailable': f'no trained parameters at {os.path.relpath(path, ROOT)} '
                               '(python -m lcode3d_b200.train_predictor writes them)'}
    cfg = make_config(args.grid, 'fp64')
    N = cfg.grid_steps
    A = GRIDS[args.grid][2]
    pr = P.FieldPredictor.load(path, grid_steps=N)
    K, W = args.steps, args.warmup

    def advance(sim, learned):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if learned:
            P.learned_steps(sim, pr, W, args.tol, args.verify_every, 0, False)
        else:
            for _ in range(W):
                sim.step_plain()
        torch.cuda.synchronize()
        ev0.record()
        if learned:
            ez, st = P.learned_steps(sim, pr, K, args.tol, args.verify_every, 0, True)
        else:
            ez = []
            for _ in range(K):
                sim.step_plain()
                ez.append(sim.state.Ez[N // 2, N // 2].clone())
            st = None
        ev1.record()
        torch.cuda.synchronize()
        return ev0.elapsed_time(ev1), torch.stack(ez).cpu().numpy(), st

    sims = []
    for _ in range(2):
        sim = P.Stepper(cfg, (A, 1.0, 1.0))
        for _ in range(args.pre):
            sim.step_plain()
        sims.append(sim)
    clocks = Clocks(dev)
    clocks.start()
    ms_l, ez_l, st = advance(sims[0], True)
    clk = clocks.stop()
    ms_p, ez_p, _ = advance(sims[1], False)
    err = float(np.abs(ez_l - ez_p).max() / max(np.abs(ez_p).max(), 1e-300))
    return {
        'metric': 'xi-steps/s', 'value': K / (ms_l * 1e-3), 'unit': 'xi-steps/s', 'n_gpus': 1, 'steps': K,
        'warmup': W, 'ms_per_step': ms_l / K, 'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
        'dtype': 'f64+bf16', 'form': 'fp64+learned',
        'data': 'synthetic (generated cold uniform plasma + axisymmetric beam; no dataset)',
        'config': {'workload': f'LCODE 3D xi step, {N}x{N} grid, learned first pass (U-Net, tcgen05) with '
                               f'periodic verification, tol {args.tol:g}, every {args.verify_every} steps',
                   'grid_steps': N, 'start_xi_step': args.pre, 'weights': os.path.relpath(path, ROOT),
                   'l2': 'not flushed', 'parallelism': 'single GPU'},
        'learned': st, 'plain_same_steps': {'value': K / (ms_p * 1e-3), 'ms_per_step': ms_p / K},
        'ez_max_rel_err_vs_plain': err, 'clocks': clk,
    }


def run_reference(args):
    threads = cpu_threads()
    K = max(1, min(args.steps, args.ref_max_steps))
    W = max(0, min(args.warmup, 10))   # untimed warm-up steps (CPU steps are slow: at most 10)
    v = time_oracle(args.grid, K, threads, args.pre, W)
    cfg = make_config(args.grid, 'fp64')
    N = cfg.grid_steps
    return {
        'impl': 'reference', 'metric': METRIC, 'value': v, 'unit': 'xi-steps/s', 'n_gpus': 0,
        'steps': K, 'warmup': W, 'ms_per_step': 1e3 / v, 'higher_is_better': True,
        'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64',
        'data': 'synthetic (generated cold uniform plasma + axisymmetric beam; no dataset)',
        'config': {'workload': f'LCODE 3D xi step, {N}x{N} grid, h={cfg.grid_step_size}, '
                               f'xi_step={cfg.xi_step_size}, coarseness 3 / fineness 2, A={GRIDS[N][2]}, '
                               'fp64 field solvers', 'grid_steps': N, 'start_xi_step': args.pre,
                   'beam': 'evaluated before the timed loop'},
        'cpu_baseline': {'value': v, 'unit': 'xi-steps/s', 'cores': threads, 'kind': 'port',
                         'sample': f'{K} xi steps of the {N}^2 workload from xi step {args.pre + W} '
                                   f'(advanced there untimed; reference algorithm: numpy + scipy.fft, '
                                   'particle kernels in C/OpenMP)'},
        'e2e': {'value': v, 'unit': 'xi-steps/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=100)
    ap.add_argument('--warmup', type=int, default=5)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--precision', default='fp64', choices=['fp64', 'mixed', 'fft32', 'tf32'])
    ap.add_argument('--fp64-transform', default='auto', choices=['auto', 'fft', 'dense'])
    ap.add_argument('--slices', type=int, default=0,
                    help='slices per operand of the tensor-core transforms (0: 4 for mixed, 3 for tf32)')
    ap.add_argument('--grid', type=int, default=641, choices=sorted(GRIDS))
    ap.add_argument('--pre', type=int, default=400, help='untimed steps into the beam')
    ap.add_argument('--cpu-steps', type=int, default=16, help='oracle steps for cpu_baseline')
    ap.add_argument('--ref-max-steps', type=int, default=40)
    ap.add_argument('--scan', type=int, default=0,
                    help='batched parameter scan of this many simulations instead of the single-grid workload')
    ap.add_argument('--seed', type=int, default=2025, help='seed of the scan draws')
    ap.add_argument('--scan-deposit', default='branches', choices=['branches', 'multi'],
                    help='scan: depositions per simulation on graph branches, or one launch over all')
    ap.add_argument('--learned', nargs='?', const='default', default=None,
                    help='learned first pass with these trained parameters (.npz; default: the packaged ones)')
    ap.add_argument('--tol', type=float, default=1e-6, help='learned: verification tolerance on max|pred - F1| / max|F1|')
    ap.add_argument('--verify-every', type=int, default=10, help='learned: steps between verifications')
    ap.add_argument('--accuracy-table', action='store_true',
                    help='error of the reduced-precision forms against float64 over a long run')
    ap.add_argument('--accuracy-steps', default='500,1500,3000', help='accuracy table: steps to report')
    ap.add_argument('--forms', default='fft32,mixed_s4,mixed_s5', help='accuracy table: forms to compare')
    args = ap.parse_args()
    if args.accuracy_table:
        print(json.dumps(run_accuracy_table(args)), flush=True)
        return
    if args.warmup < 3 and args.impl == 'ours':
        args.warmup = 3

    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    if args.impl == 'reference':
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get('LOCAL_RANK', 0)))
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=300))
    if args.learned:
        if rank == 0:
            print(json.dumps(run_learned_bench(args)), flush=True)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    if args.scan:
        out = run_scan(args, rank, world, dist)
        if rank == 0:
            print(json.dumps(out), flush=True)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    out = run_ours(args, rank, world, dist)
    if rank == 0:
        threads = 1
        v = time_oracle(args.grid, args.cpu_steps, threads, 0)
        out['cpu_baseline'] = {
            'value': v, 'unit': 'xi-steps/s', 'cores': threads, 'kind': 'port',
            'sample': f'{args.cpu_steps} xi steps of the {args.grid}^2 workload from its initial state '
                      '(beams evaluated before the timed loop), oracle restatement of the reference '
                      '(numpy + scipy.fft, particle kernels in C), 1 thread'}
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == '__main__':
    main()
