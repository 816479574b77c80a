#!/usr/bin/env python3
"""Generate the golden input/output vectors of the reference ``lcode.py``.

This script is test infrastructure. It runs the UNMODIFIED algorithm of the
reference LCODE 3D (``lcode.py``, a single Python module whose GPU work goes
through cupy + cuFFT and two ``numba.cuda`` kernels) on the CPU, by loading
the module text with a handful of mechanical substitutions:

* ``cupy`` is replaced by a namespace backed by numpy (``cp.fft.rfft2`` ->
  ``numpy.fft.rfft2``, ``cp.memoize`` -> ``functools.lru_cache``,
  ``cp.cuda.Device`` -> a no-op context manager);
* ``matplotlib`` is stubbed (only used for PNG diagnostics);
* ``@numba.jit(inline=True)`` -> ``@numba.njit`` (numba >= 0.5x rejects
  ``inline=True`` at call time);
* ``numba.cuda.atomic.add(a, (i, j), v)`` -> ``a[i, j] += v``;
* the two ``@numba.cuda.jit`` kernels become ``@numba.njit`` bodies taking the
  thread index as an argument, launched by a serial loop over all
  ``blocks * 32`` thread ids (so the deposition order is the ascending fine
  particle index: deterministic);
* ``numba.cuda.synchronize()`` -> no-op.

Everything else (init, plasma layout, pusher, deposition arithmetic, the
padded-rFFT DST/DCT solvers, the predictor-corrector ``step``) is the
reference's own code.

The reference only exists in the build container, so the vectors are
committed as ``.npz`` fixtures next to this script and the tests read those.

Usage:  python tests/golden/make_golden.py --ref <reference checkout> [--which all|stages|cfg1|cfg2]
        (or set LCODE_REFERENCE to the checkout instead of passing --ref)

        python tests/golden/make_golden.py --ref R --which cfg2full [--resume-dir D]
        python tests/golden/make_golden.py --ref R --which cfg2full-reversed --out REV.npz [--resume-dir D2]
        python tests/golden/make_golden.py --which cfg2floor --out REV.npz

``cfg2full`` runs the 641^2 production configuration for its whole 3000
steps (several CPU hours) twice: once in the serial deposition order and once
with the deposition's thread ids visited in reverse. The second run stands in
for another order of the reference's float64 atomics, and the difference of
the two is the order-sensitivity floor stored beside the fixture.
"""
import argparse
import functools
import os
import sys
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


# --------------------------------------------------------------------------
# Loading the reference with shims
# --------------------------------------------------------------------------

def _fake_cupy():
    cp = types.ModuleType('cupy')
    for name in dir(np):
        if not name.startswith('__'):
            setattr(cp, name, getattr(np, name))
    cp.fft = np.fft

    def memoize(*_a, **_k):
        def deco(f):
            return functools.lru_cache(maxsize=None)(f)
        return deco
    cp.memoize = memoize

    class _Device:
        def __init__(self, *_a):
            pass

        def __enter__(self):
            return self

        def __exit__(self, *_a):
            return False
    cuda = types.ModuleType('cupy.cuda')
    cuda.Device = _Device
    cp.cuda = cuda
    return cp


def _fake_matplotlib():
    mpl = types.ModuleType('matplotlib')
    plt = types.ModuleType('matplotlib.pyplot')
    plt.imsave = lambda *a, **k: None
    mpl.pyplot = plt
    return mpl, plt


def load_reference(ref_dir, reverse_deposit=False):
    """Return the reference ``lcode`` module running on numpy + numba (CPU).

    With ``reverse_deposit`` the deposition kernel's thread ids are visited
    from the last to the first (another order of the same float64 adds)."""
    import numba
    src = open(os.path.join(ref_dir, 'lcode.py')).read()

    def sub(old, new, count=None):
        nonlocal src
        n = src.count(old)
        if n == 0 or (count is not None and n != count):
            raise RuntimeError(f'reference text changed: {old!r} x{n}')
        src = src.replace(old, new)

    sub('@numba.jit(inline=True)', '@numba.njit', 5)
    # atomic.add(a, (i + di, j + dj), v) -> a[i + di, j + dj] += v
    import re
    pat = re.compile(r'numba\.cuda\.atomic\.add\((\w+), \(([^)]*)\), ([^)]*)\)')
    src, n = pat.subn(r'\1[\2] += \3', src)
    assert n == 9, n
    sub('@numba.cuda.jit\ndef deposit_kernel(',
        '@numba.njit\ndef deposit_kernel_body(_tid, ', 1)
    sub('@numba.cuda.jit\ndef move_smart_kernel(',
        '@numba.njit\ndef move_smart_kernel_body(_tid, ', 1)
    sub('numba.cuda.grid(1)', '_tid', 2)
    sub('numba.cuda.synchronize()', 'None')
    src += '''

def _make_launcher(body, reverse=False):
    @numba.njit
    def _loop(n, args):
        for t in range(n):
            body(n - 1 - t if reverse else t, *args)

    class _Launcher:
        def __getitem__(self, cfg):
            blocks, threads = cfg
            return lambda *args: _loop(blocks * threads, args)
    return _Launcher()


deposit_kernel = _make_launcher(deposit_kernel_body, _REVERSE_DEPOSIT)
move_smart_kernel = _make_launcher(move_smart_kernel_body)
'''
    saved = {k: sys.modules.get(k) for k in ('cupy', 'matplotlib', 'matplotlib.pyplot')}
    mpl, plt = _fake_matplotlib()
    sys.modules['cupy'] = _fake_cupy()
    sys.modules['matplotlib'] = mpl
    sys.modules['matplotlib.pyplot'] = plt
    try:
        mod = types.ModuleType('lcode_reference')
        mod.__file__ = os.path.join(ref_dir, 'lcode.py')
        mod._REVERSE_DEPOSIT = bool(reverse_deposit)
        exec(compile(src, mod.__file__, 'exec'), mod.__dict__)
    finally:
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v
    assert mod.numba is numba
    return mod


# --------------------------------------------------------------------------
# Configurations
# --------------------------------------------------------------------------

def make_config(grid_steps, grid_step_size, xi_step_size, xi_steps,
                amplitude, sigma_r=1.0, length_factor=1.0):
    """A config module object with the reference's attribute names.

    The beam is the axisymmetric electron driver
    rho_b = A exp(-r^2 / (2 sigma_r^2)) * 0.5 (1 - cos(sqrt(pi/2) xi / L))
    for 0 <= xi <= 2 sqrt(2 pi) L (L = length_factor), else 0,
    with xi = xi_i * xi_step_size.
    """
    c = types.SimpleNamespace()
    c.grid_steps = grid_steps
    c.grid_step_size = grid_step_size
    c.xi_step_size = xi_step_size
    c.xi_steps = xi_steps
    c.diagnostics_each_N_steps = 10 ** 9
    c.field_solver_subtraction_trick = 1
    c.field_solver_variant_A = True
    c.reflect_padding_steps = 5
    c.plasma_padding_steps = 10
    c.plasma_coarseness = 3
    c.plasma_fineness = 2
    c.gpu_index = 0

    def beam(xi_i, x, y):
        xi = xi_i * xi_step_size
        if xi < 0 or xi > 2 * np.sqrt(2 * np.pi) * length_factor:
            return 0
        r2 = x ** 2 + y ** 2
        return (amplitude * np.exp(-r2 / (2 * sigma_r ** 2)) * 0.5 *
                (1 - np.cos(np.sqrt(np.pi / 2) * xi / length_factor)))
    c.beam = beam
    return c


def beam_array(config, xi_i, xs, ys):
    b = config.beam(xi_i, xs, ys)
    N = config.grid_steps
    return np.broadcast_to(np.asarray(b, dtype=np.float64), (N, N)).copy()


def state_dict(s):
    return {k: np.array(getattr(s, k)) for k in
            ('x_offt', 'y_offt', 'px', 'py', 'pz', 'Ex', 'Ey', 'Ez',
             'Bx', 'By', 'Bz', 'ro', 'jx', 'jy', 'jz')}


# --------------------------------------------------------------------------
# Per-function vectors on a small grid with a perturbed state
# --------------------------------------------------------------------------

def gen_stages(lc, out):
    cfg = make_config(41, 0.1, 0.05, 10, amplitude=0.3)
    xs, ys, const, virt, state = lc.init(cfg)
    rng = np.random.default_rng(20190501)
    N = cfg.grid_steps
    Nc = const.m.shape[0]
    h = cfg.grid_step_size

    # A perturbed, physically plausible prev state that exercises every
    # term: offsets, momenta, all six fields, densities, and particles that
    # cross the reflection boundary in both the estimate and the pusher.
    prev = {}
    prev['x_offt'] = rng.uniform(-0.8, 0.8, (Nc, Nc)) * h
    prev['y_offt'] = rng.uniform(-0.8, 0.8, (Nc, Nc)) * h
    prev['px'] = rng.normal(0, 0.05, (Nc, Nc))
    prev['py'] = rng.normal(0, 0.05, (Nc, Nc))
    prev['pz'] = rng.normal(0, 0.05, (Nc, Nc))
    # push the outer ring of coarse particles towards/over the reflect
    # boundary; reflect_boundary = h * (N / 2 - 5) = 1.55 here
    rb = cfg.reflect_boundary
    x_init = np.array(const.x_init)
    y_init = np.array(const.y_init)
    edge = rng.random((Nc, Nc)) < 0.3
    for arr, init, mom in ((prev['x_offt'], x_init, prev['px']),
                           (prev['y_offt'], y_init, prev['py'])):
        sgn = np.sign(init + 1e-9)
        target = sgn * (rb - rng.uniform(-0.02, 0.03, (Nc, Nc)))
        arr[edge] = (target - init)[edge]
        mom[edge] = (sgn * rng.uniform(0.2, 0.6, (Nc, Nc)))[edge]
    # one particle exactly on the boundary exercises '>=' vs '>'
    prev['x_offt'][0, 0] = -rb - x_init[0, 0]
    prev['px'][0, 0] = 0.0

    def smooth_field(scale):
        f = rng.normal(0, scale, (N, N))
        k = np.ones(5) / 5
        for ax in (0, 1):
            f = np.apply_along_axis(lambda v: np.convolve(v, k, 'same'), ax, f)
        f[0, :] = f[-1, :] = f[:, 0] = f[:, -1] = 0
        return f
    for name in ('Ex', 'Ey', 'Ez', 'Bx', 'By', 'Bz'):
        prev[name] = smooth_field(0.2)
    for name in ('ro', 'jx', 'jy', 'jz'):
        prev[name] = smooth_field(0.05)
    beam_ro = beam_array(cfg, 40, xs, ys)

    g = {}
    g['grid_steps'] = N
    g['grid_step_size'] = h
    g['xi_step_size'] = cfg.xi_step_size
    g['reflect_boundary'] = cfg.reflect_boundary
    for k in ('m', 'q', 'x_init', 'y_init', 'ro_initial'):
        g['const_' + k] = np.array(getattr(const, k))
    for k in ('influence_prev', 'influence_next', 'indices_prev',
              'indices_next', 'fine_grid'):
        g['virt_' + k] = np.array(getattr(virt, k))
    g['xs'] = np.array(xs).ravel()
    for k, v in prev.items():
        g['prev_' + k] = v
    g['beam_ro'] = beam_ro

    P = types.SimpleNamespace(**prev)
    est_x, est_y = lc.move_estimate_wo_fields(
        cfg, const.m, const.x_init, const.y_init, P.x_offt, P.y_offt,
        P.px, P.py, P.pz)
    g['est_x_offt'], g['est_y_offt'] = est_x, est_y
    mx, my, mpx, mpy, mpz = lc.move_smart(
        cfg, const.m, const.q, const.x_init, const.y_init,
        P.x_offt, P.y_offt, est_x, est_y, P.px, P.py, P.pz,
        P.Ex, P.Ey, P.Ez, P.Bx, P.By, P.Bz)
    for k, v in zip(('x_offt', 'y_offt', 'px', 'py', 'pz'), (mx, my, mpx, mpy, mpz)):
        g['move_' + k] = v
    ro, jx, jy, jz = lc.deposit(cfg, const.ro_initial, mx, my, const.m,
                                const.q, mpx, mpy, mpz, virt)
    for k, v in zip(('ro', 'jx', 'jy', 'jz'), (ro, jx, jy, jz)):
        g['dep_' + k] = v
    Ex, Ey, Bx, By = lc.calculate_Ex_Ey_Bx_By(
        cfg, P.Ex, P.Ey, P.Bx, P.By, beam_ro, ro, jx, jy, jz, P.jx, P.jy)
    for k, v in zip(('Ex', 'Ey', 'Bx', 'By'), (Ex, Ey, Bx, By)):
        g['fld_' + k] = v
    g['fld_Ez'] = lc.calculate_Ez(cfg, jx, jy)
    g['fld_Bz'] = lc.calculate_Bz(cfg, jx, jy)
    # Laplace variant of the transverse solver (subtraction trick off)
    cfg0 = make_config(41, 0.1, 0.05, 10, amplitude=0.3)
    cfg0.field_solver_subtraction_trick = 0
    lc.init(cfg0)
    Ex0, Ey0, Bx0, By0 = lc.calculate_Ex_Ey_Bx_By(
        cfg0, P.Ex, P.Ey, P.Bx, P.By, beam_ro, ro, jx, jy, jz, P.jx, P.jy)
    for k, v in zip(('Ex', 'Ey', 'Bx', 'By'), (Ex0, Ey0, Bx0, By0)):
        g['fld0_' + k] = v

    # one full step from the perturbed state, both field-solver variants
    new = lc.step(cfg, const, virt, P, beam_ro)
    for k, v in state_dict(new).items():
        g['step_' + k] = v
    cfgB = make_config(41, 0.1, 0.05, 10, amplitude=0.3)
    cfgB.field_solver_variant_A = False
    lc.init(cfgB)
    newB = lc.step(cfgB, const, virt, P, beam_ro)
    for k, v in state_dict(newB).items():
        g['stepB_' + k] = v

    # the transforms on their own
    a = rng.normal(size=(N - 2, N - 2))
    g['tr_dst_in'] = a
    g['tr_dst_out'] = lc.dst2d(a)
    b = rng.normal(size=(N, N))
    g['tr_dct_in'] = b
    g['tr_dct_out'] = lc.dct2d(b)
    c = rng.normal(size=(N - 2, N))
    g['tr_mix_in'] = c
    g['tr_mix_out'] = lc.mix2d(c)
    np.savez_compressed(out, **g)


# --------------------------------------------------------------------------
# Whole runs
# --------------------------------------------------------------------------

def run(lc, cfg, steps, record=None, snap_every=None):
    xs, ys, const, virt, state = lc.init(cfg)
    N = cfg.grid_steps
    ez = []
    snaps = {}
    t0 = time.time()
    for xi_i in range(steps):
        b = beam_array(cfg, xi_i, xs, ys)
        state = lc.step(cfg, const, virt, state, b)
        ez.append(float(state.Ez[N // 2, N // 2]))
        if record is not None:
            record(xi_i, state, snaps)
    dt = time.time() - t0
    return const, virt, state, np.array(ez), snaps, dt


def gen_cfg1(lc, out):
    # 161^2, h=0.05, dxi=0.05, 300 steps, A=0.05, sigma_r=1
    cfg = make_config(161, 0.05, 0.05, 300, amplitude=0.05)
    keep = ('Ex', 'Ey', 'Ez', 'Bz', 'ro', 'jz')

    def record(xi_i, st, snaps):
        if xi_i + 1 in (1, 100):
            for k in keep:
                snaps[f's{xi_i + 1}_{k}'] = np.array(getattr(st, k))
    const, virt, state, ez, snaps, dt = run(lc, cfg, 300, record)
    g = dict(snaps)
    g['Ez00'] = ez
    for k in keep + ('x_offt', 'y_offt', 'px', 'py', 'pz'):
        g['final_' + k] = np.array(getattr(state, k))
    g['seconds'] = dt
    np.savez_compressed(out, **g)
    print(f'cfg1: 300 steps in {dt:.1f} s', flush=True)


def gen_cfg2(lc, out, steps):
    # 641^2, h=0.025, dxi=0.005, A=0.5, sigma_r=1; the first `steps` steps
    cfg = make_config(641, 0.025, 0.005, 3000, amplitude=0.5)
    N = cfg.grid_steps

    def summary(prefix, st, g):
        for k, v in state_dict(st).items():
            if v.shape == (N, N):
                g[prefix + 'axis_' + k] = v[N // 2, :].copy()
                g[prefix + 'diag_' + k] = np.diagonal(v).copy()
            g[prefix + 'sum_' + k] = v.sum()
            g[prefix + 'abssum_' + k] = np.abs(v).sum()
            g[prefix + 'maxabs_' + k] = np.abs(v).max()

    def record(xi_i, st, snaps):
        if xi_i + 1 == 2:
            summary('s2_', st, snaps)
    const, virt, state, ez, snaps, dt = run(lc, cfg, steps, record)
    g = {'Ez00': ez, 'seconds': dt, 'steps': steps}
    g.update(snaps)
    summary('', state, g)
    g['ro_initial_sum'] = np.array(const.ro_initial).sum()
    np.savez_compressed(out, **g)
    print(f'cfg2: {steps} steps in {dt:.1f} s', flush=True)


FULL_SNAPSHOTS = (500, 1000, 1500, 3000)


def _rows_summary(prefix, st, g):
    """Middle row and main diagonal of every state array (grids N x N and
    coarse particle arrays Nc x Nc), plus its sum, sum of moduli and maximum
    modulus."""
    for k, v in state_dict(st).items():
        n = v.shape[0]
        g[prefix + 'axis_' + k] = v[n // 2, :].copy()
        g[prefix + 'diag_' + k] = np.diagonal(v).copy()
        g[prefix + 'sum_' + k] = v.sum()
        g[prefix + 'abssum_' + k] = np.abs(v).sum()
        g[prefix + 'maxabs_' + k] = np.abs(v).max()


def gen_cfg2_full(lc, out, resume_dir=None):
    """The whole 641^2 production run (h=0.025, dxi=0.005, A=0.5, 3000 steps):
    the Ez(0,0) history and row summaries at FULL_SNAPSHOTS. With
    ``resume_dir`` the state is saved there every 250 steps and a saved state
    is picked up again, so an interrupted run continues where it stopped."""
    cfg = make_config(641, 0.025, 0.005, 3000, amplitude=0.5)
    N = cfg.grid_steps
    steps = 3000
    xs, ys, const, virt, state = lc.init(cfg)
    ez = np.zeros(steps)
    g = {}
    start = 0
    ck = os.path.join(resume_dir, 'cfg2full_ck.npz') if resume_dir else None
    if ck and os.path.exists(ck):
        z = np.load(ck)
        start = int(z['next_step'])
        ez[:start] = z['ez'][:start]
        g = {k[5:]: z[k] for k in z.files if k.startswith('snap_')}
        state = lc.GPUArrays(**{k: z['st_' + k] for k in state_dict(state)})
        print(f'cfg2full: resumed at step {start}', flush=True)
    t0 = time.time()
    for xi_i in range(start, steps):
        b = beam_array(cfg, xi_i, xs, ys)
        state = lc.step(cfg, const, virt, state, b)
        ez[xi_i] = float(state.Ez[N // 2, N // 2])
        if xi_i + 1 in FULL_SNAPSHOTS:
            _rows_summary(f's{xi_i + 1}_', state, g)
        if ck and (xi_i + 1) % 250 == 0 and xi_i + 1 < steps:
            d = {'st_' + k: v for k, v in state_dict(state).items()}
            d.update({'snap_' + k: v for k, v in g.items()})
            np.savez(ck + '.tmp.npz', next_step=xi_i + 1, ez=ez, **d)
            os.replace(ck + '.tmp.npz', ck)
            print(f'cfg2full: step {xi_i + 1}, {time.time() - t0:.0f} s', flush=True)
    g['Ez00'] = ez
    g['steps'] = steps
    g['snapshots'] = np.array(FULL_SNAPSHOTS)
    np.savez_compressed(out, **g)
    print(f'cfg2full: {steps} steps, {time.time() - t0:.1f} s in this process', flush=True)


def gen_cfg2_floor(serial, reversed_, out):
    """Order-sensitivity floor of the full run: for every recorded quantity,
    the largest difference between the serial and the reversed deposition
    order relative to the quantity's scale (max modulus of the serial
    values). Written into the serial fixture as ``floor_<key>``."""
    a = dict(np.load(serial))
    b = np.load(reversed_)
    for k in list(a):
        if k in ('steps', 'snapshots') or k.startswith('floor_'):
            continue
        x, y = np.asarray(a[k], dtype=np.float64), np.asarray(b[k], dtype=np.float64)
        scale = max(np.abs(x).max(), 1e-300)
        a['floor_' + k] = np.abs(x - y).max() / scale
    np.savez_compressed(out, **a)
    worst = sorted(((float(v), k) for k, v in a.items() if k.startswith('floor_')), reverse=True)
    for v, k in worst[:12]:
        print(f'{k}: {v:.2e}')


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--ref', default=os.environ.get('LCODE_REFERENCE'),
                    help='reference checkout holding lcode.py (or LCODE_REFERENCE)')
    ap.add_argument('--which', default='all')
    ap.add_argument('--cfg2-steps', type=int, default=30)
    ap.add_argument('--resume-dir', default=None,
                    help='cfg2full: where to keep the resumable state of the run')
    ap.add_argument('--out', default=None, help='cfg2full: output file')
    a = ap.parse_args()
    full = os.path.join(HERE, 'run_n641_full.npz')
    if a.which == 'cfg2floor':
        # combine a serial and a reversed run (both written by cfg2full)
        gen_cfg2_floor(full, a.out, full)
        return
    if not a.ref:
        ap.error('--ref (or LCODE_REFERENCE) is required')
    if a.which == 'cfg2full-reversed':
        lc = load_reference(a.ref, reverse_deposit=True)
        gen_cfg2_full(lc, a.out, a.resume_dir)
        return
    lc = load_reference(a.ref)
    if a.which in ('all', 'stages'):
        gen_stages(lc, os.path.join(HERE, 'stages_n41.npz'))
        print('stages done', flush=True)
    if a.which in ('all', 'cfg1'):
        gen_cfg1(lc, os.path.join(HERE, 'run_n161.npz'))
    if a.which in ('all', 'cfg2'):
        gen_cfg2(lc, os.path.join(HERE, 'run_n641_head.npz'), a.cfg2_steps)
    if a.which == 'cfg2full':
        gen_cfg2_full(lc, a.out or full, a.resume_dir)


if __name__ == '__main__':
    main()
