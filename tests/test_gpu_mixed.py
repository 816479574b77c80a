"""Mixed-precision field solvers (split-BF16 tcgen05 GEMMs, FP32 accumulate,
float64 combination) against the float64 path and the reference.

The tolerances are the error levels of the split scheme with S slices per
operand (exact FP32 accumulation of the digit levels; truncation ~2^-7S of
the row maxima, amplified by the four transform stages), with headroom."""
import os

import numpy as np
import pytest

torch = pytest.importorskip('torch')

from conftest import GOLDEN  # noqa: E402
from make_golden import beam_array, make_config  # noqa: E402
from oracle import lcode_oracle as O  # noqa: E402

pytestmark = pytest.mark.gpu

FIELD_TOL = {1: 0.25, 2: 1e-2, 3: 1e-4, 4: 3e-6, 5: 1e-7, 6: 1e-8}


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


@pytest.mark.parametrize('S,N', [(S, N) for S in (2, 3, 4, 5) for N in (41, 161, 641)] + [(1, 161), (6, 161), (6, 641)])
def test_mixed_solvers_vs_fp64(L, N, S):
    rng = np.random.default_rng(100 * N + S)
    h = 16 / (N - 1)
    ins = [torch.from_numpy(rng.normal(size=(N, N))).cuda() for _ in range(11)]
    cfg64 = make_config(N, h, 0.01, 10, amplitude=0.1)
    cfgm = make_config(N, h, 0.01, 10, amplitude=0.1)
    cfgm.lc3d_precision = 'mixed'
    cfgm.lc3d_mixed_slices = S
    ref = solve_all(L, cfg64, ins)
    got = solve_all(L, cfgm, ins)
    errs = {k: rel(a, b) for k, a, b in zip(('Ex', 'Ey', 'Bx', 'By', 'Ez', 'Bz'), got, ref)}
    print(f'N={N} S={S} relative errors vs float64: ' +
          ' '.join(f'{k}={v:.2e}' for k, v in errs.items()))
    for k, v in errs.items():
        assert v < FIELD_TOL[S], (k, v)


def test_mixed_step_fixture(L):
    """One full step (41^2) in mixed precision against the reference."""
    g = np.load(os.path.join(GOLDEN, 'stages_n41.npz'))
    cfg = make_config(41, 0.1, 0.05, 10, amplitude=0.3)
    cfg.lc3d_precision = 'mixed'
    cfg.lc3d_mixed_slices = 5
    xs, ys, c, virt, _ = L.init(cfg)
    P = {k[5:]: torch.from_numpy(g[k]).cuda() for k in g.files if k.startswith('prev_')}
    import types
    new = L.step(cfg, c, virt, types.SimpleNamespace(**P), torch.from_numpy(g['beam_ro']).cuda())
    for k in ('x_offt', 'y_offt', 'px', 'py', 'pz', 'Ex', 'Ey', 'Ez', 'Bx', 'By', 'Bz', 'ro', 'jx', 'jy', 'jz'):
        assert rel(getattr(new, k), g['step_' + k]) < 1e-7, k


@pytest.mark.parametrize('S', [4, 5])
def test_mixed_run_n161(L, S):
    """300 steps of the 161^2 run in mixed precision: on-axis Ez history and
    final fields against the reference (float64) vectors."""
    g = np.load(os.path.join(GOLDEN, 'run_n161.npz'))
    cfg = make_config(161, 0.05, 0.05, 300, amplitude=0.05)
    cfg.lc3d_precision = 'mixed'
    cfg.lc3d_mixed_slices = S
    xs, ys, const, virt, st = L.init(cfg)
    ez = []
    for i in range(300):
        st = L.step(cfg, const, virt, st, beam_array(cfg, i, xs, ys))
        ez.append(float(st.Ez[80, 80]))
    e = rel(np.array(ez), g['Ez00'])
    errs = {k: rel(getattr(st, k), g['final_' + k]) for k in ('Ex', 'Ey', 'Ez', 'Bz', 'ro', 'jz')}
    print(f'161^2 x 300 steps, S={S}: Ez00 history {e:.2e}; final ' +
          ' '.join(f'{k}={v:.2e}' for k, v in errs.items()))
    assert e < 1e-6
    for k, v in errs.items():
        assert v < 1e-4, (k, v)


@pytest.mark.parametrize('S', [2, 3])
@pytest.mark.parametrize('N', [41, 161, 641])
def test_tf32_solvers_vs_fp64(L, N, S):
    """The split-TF32 transforms (tcgen05 kind::tf32, 10-bit digits): the
    FP32 accumulation is not exact for these digits, so besides the
    truncation (2^-10S of the row maxima) every stage carries FP32 rounding
    of its sums; the bound here is that level with the stages'
    amplification and headroom."""
    rng = np.random.default_rng(300 * N + S)
    h = 16 / (N - 1)
    ins = [torch.from_numpy(rng.normal(size=(N, N))).cuda() for _ in range(11)]
    cfg64 = make_config(N, h, 0.01, 10, amplitude=0.1)
    cfgt = make_config(N, h, 0.01, 10, amplitude=0.1)
    cfgt.lc3d_precision = 'tf32'
    cfgt.lc3d_mixed_slices = S
    ref = solve_all(L, cfg64, ins)
    got = solve_all(L, cfgt, ins)
    errs = {k: rel(a, b) for k, a, b in zip(('Ex', 'Ey', 'Bx', 'By', 'Ez', 'Bz'), got, ref)}
    print(f'N={N} tf32 S={S} relative errors vs float64: ' +
          ' '.join(f'{k}={v:.2e}' for k, v in errs.items()))
    for k, v in errs.items():
        assert v < 1e-3, (k, v)
