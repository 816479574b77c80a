"""Float32-transform field solvers (lc3d_precision = 'fft32': the four FFT
row passes of every solve in float32, float32 intermediates and
eigenvalues; right-hand sides, field outputs, averaging and particles in
float64) against the float64 path and the reference.

Tolerances: a float32 FFT of length P = 2(N - 1) is accurate to a few
float32 ulps times log2(P) of the row maximum; four passes and the
eigenvalue scaling keep a solve within ~1e-6 of the field maximum. Over a
run the errors feed back through the particles; the on-axis Ez history and
the Ez field stay within 1e-6 of their maxima."""
import os

import numpy as np
import pytest

torch = pytest.importorskip('torch')

from conftest import GOLDEN  # noqa: E402
from make_golden import beam_array, make_config  # noqa: E402
from oracle import lcode_oracle as O  # noqa: E402

pytestmark = pytest.mark.gpu


def rel(a, b):
    return O.relative_error(a.cpu().numpy() if isinstance(a, torch.Tensor) else a,
                            b.cpu().numpy() if isinstance(b, torch.Tensor) else b)


@pytest.fixture(scope='module')
def L():
    if not torch.cuda.is_available():
        pytest.skip('no GPU')
    import lcode3d_b200 as L
    L.lcode.check_errors = True
    return L


def solve_all(L, cfg, ins):
    F = L.calculate_Ex_Ey_Bx_By(cfg, *ins)
    Ez = L.calculate_Ez(cfg, ins[6], ins[7])
    Bz = L.calculate_Bz(cfg, ins[6], ins[7])
    torch.cuda.synchronize()
    return (*F, Ez, Bz)


@pytest.mark.parametrize('N', [41, 161, 641])
def test_fft32_solvers_vs_fp64(L, N):
    rng = np.random.default_rng(7 * N)
    h = 16 / (N - 1)
    ins = [torch.from_numpy(rng.normal(size=(N, N))).cuda() for _ in range(11)]
    cfg64 = make_config(N, h, 0.01, 10, amplitude=0.1)
    cfg32 = make_config(N, h, 0.01, 10, amplitude=0.1)
    cfg32.lc3d_precision = 'fft32'
    ref = solve_all(L, cfg64, ins)
    got = solve_all(L, cfg32, ins)
    errs = {k: rel(a, b) for k, a, b in zip(('Ex', 'Ey', 'Bx', 'By', 'Ez', 'Bz'), got, ref)}
    print(f'N={N} fft32 relative errors vs float64: ' + ' '.join(f'{k}={v:.2e}' for k, v in errs.items()))
    for k, v in errs.items():
        assert v < 2e-5, (k, v)


def test_fft32_step_fixture(L):
    """One full step (41^2) with float32 transforms against the reference."""
    g = np.load(os.path.join(GOLDEN, 'stages_n41.npz'))
    cfg = make_config(41, 0.1, 0.05, 10, amplitude=0.3)
    cfg.lc3d_precision = 'fft32'
    xs, ys, c, virt, _ = L.init(cfg)
    P = {k[5:]: torch.from_numpy(g[k]).cuda() for k in g.files if k.startswith('prev_')}
    import types
    new = L.step(cfg, c, virt, types.SimpleNamespace(**P), torch.from_numpy(g['beam_ro']).cuda())
    errs = {k: rel(getattr(new, k), g['step_' + k])
            for k in ('x_offt', 'y_offt', 'px', 'py', 'pz', 'Ex', 'Ey', 'Ez', 'Bx', 'By', 'Bz', 'ro', 'jx', 'jy', 'jz')}
    print('41^2 step, fft32: ' + ' '.join(f'{k}={v:.1e}' for k, v in errs.items()))
    for k, v in errs.items():
        assert v < 1e-5, (k, v)


def test_fft32_run_n161(L):
    """300 steps of the 161^2 run with float32 transforms: on-axis Ez
    history and final fields against the reference (float64) vectors."""
    g = np.load(os.path.join(GOLDEN, 'run_n161.npz'))
    cfg = make_config(161, 0.05, 0.05, 300, amplitude=0.05)
    cfg.lc3d_precision = 'fft32'
    xs, ys, const, virt, st = L.init(cfg)
    ez = []
    for i in range(300):
        st = L.step(cfg, const, virt, st, beam_array(cfg, i, xs, ys))
        ez.append(float(st.Ez[80, 80]))
    e = rel(np.array(ez), g['Ez00'])
    errs = {k: rel(getattr(st, k), g['final_' + k]) for k in ('Ex', 'Ey', 'Ez', 'Bz', 'ro', 'jz')}
    print(f'161^2 x 300 steps, fft32: Ez00 history {e:.2e}; final ' +
          ' '.join(f'{k}={v:.2e}' for k, v in errs.items()))
    assert e < 1e-6
    assert errs['Ez'] < 1e-6
    for k, v in errs.items():
        assert v < 1e-3, (k, v)


def test_fft32_bench_workload_ez_gate(L):
    """The 641^2 production run (A = 0.5, blowout, dxi = 0.005) over its whole
    3000 steps from the initial state with float32 and float64 transforms:
    the on-axis Ez history and the final Ez field agree to 1e-6 of their
    maxima (the accuracy gate of the reduced-precision form)."""
    import bench
    N = 641
    steps = 3000
    hist, last = {}, {}
    for prec in ('fp64', 'fft32'):
        cfg = bench.make_config(N, prec)
        xs, ys, const, virt, st = L.init(cfg)
        ez = []
        for i in range(steps):
            st = L.step(cfg, const, virt, st, bench.beam_np(cfg, i, xs, ys))
            ez.append(st.Ez[N // 2, N // 2].clone())
        hist[prec] = torch.stack(ez).cpu().numpy()
        last[prec] = st.Ez.cpu().numpy()
    e_h = rel(hist['fft32'], hist['fp64'])
    e_f = rel(last['fft32'], last['fp64'])
    print(f'641^2 x {steps} steps, fft32 vs fp64: Ez axis history {e_h:.2e}, final Ez field {e_f:.2e}')
    assert e_h <= 1e-6
    assert e_f <= 1e-6
