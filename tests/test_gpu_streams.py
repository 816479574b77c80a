"""The field solves' FFT passes run on several streams (the field groups
Ex Ey Ez / Bx By Bz in float64, Ex Ey / Bx By / Ez Bz with float32
transforms), each group finalised on its own stream and joined before the
next push. With per-launch timing on (lc3d_profile) the same step runs on
the caller's stream alone. Every field is computed by the same kernels in
the same order either way, so the two must agree bit for bit; a missing
fork or join (a pass reading its input before the producing pass finished,
a push reading fields before their finalize) shows up as a difference."""
import ctypes

import pytest

torch = pytest.importorskip('torch')

from make_golden import beam_array, make_config  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def L():
    if not torch.cuda.is_available():
        pytest.skip('no GPU')
    import lcode3d_b200 as L
    L.lcode.check_errors = True
    return L


def state_tensors(L, st):
    return [getattr(st, n).clone() for n in L._lib.STATE_NAMES]


@pytest.mark.parametrize('precision', ['fp64', 'fft32'])
@pytest.mark.parametrize('N', [161, 641])
def test_multi_stream_step_matches_single_stream(L, precision, N):
    cfg = make_config(N, 16 / (N - 1), 0.01, 10, amplitude=0.5)
    cfg.lc3d_precision = precision
    xs, ys, const, virt, st = L.init(cfg)
    for i in range(8):   # into the beam, so every field is non-trivial
        st = L.step(cfg, const, virt, st, beam_array(cfg, i, xs, ys))
    beam = beam_array(cfg, 8, xs, ys)
    s = L.solver_for(cfg)
    runs = []
    for prof in (0, 1, 0):
        L._lib.check(L._lib.lib.lc3d_profile(s.ctx, prof), 'lc3d_profile')
        out = L.step(cfg, const, virt, st, beam)
        torch.cuda.synchronize()
        runs.append(state_tensors(L, out))
    L._lib.check(L._lib.lib.lc3d_profile(s.ctx, 0), 'lc3d_profile')
    for name, a, b, c in zip(L._lib.STATE_NAMES, *runs):
        assert torch.equal(a, b), f'{name}: several streams differ from one stream'
        assert torch.equal(a, c), f'{name}: several streams differ run to run'
    assert float(runs[0][L._lib.STATE_NAMES.index('Ez')].abs().max()) > 0
