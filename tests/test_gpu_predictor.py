"""The learned field predictor on the GPU: packing, the tcgen05 forward pass
and the float32 training kernels against the numpy oracle
(oracle/predictor_oracle.py), the first-pass and predicted steps against
the plain step (bit for bit when the prediction is exact), training gain
over linear extrapolation, and the verification policy of run_learned."""
import types

import numpy as np
import pytest

torch = pytest.importorskip('torch')

from make_golden import make_config  # noqa: E402
from oracle import predictor_oracle as PO  # noqa: E402

pytestmark = pytest.mark.gpu

STATE = ('x_offt', 'y_offt', 'px', 'py', 'pz', 'Ex', 'Ey', 'Ez', 'Bx', 'By', 'Bz', 'ro', 'jx', 'jy', 'jz')

# tolerances of the bf16 network against the float64 oracle that rounds to
# bf16 at the same points (rounding of float32 vs float64 sums can flip a
# bf16 value by one unit, 2^-8 relative, and such flips propagate)
FWD_MAX_TOL = 1e-2
FWD_RMS_TOL = 3e-3
GRAD_TOL = 1e-3


@pytest.fixture(scope='module')
def P():
    if not torch.cuda.is_available():
        pytest.skip('no GPU')
    import lcode3d_b200 as L
    L.lcode.check_errors = True
    from lcode3d_b200 import predictor
    return predictor


def _fields(N, seed):
    g = torch.Generator(device='cpu').manual_seed(seed)
    x = torch.linspace(-1, 1, N, dtype=torch.float64)
    base = torch.exp(-(x[:, None] ** 2 + x[None, :] ** 2) * 3)
    f1, f2 = types.SimpleNamespace(), types.SimpleNamespace()
    for k, n in enumerate(('ro', 'jx', 'jy', 'jz', 'Ex', 'Ey', 'Bx', 'By', 'Bz', 'Ez')):
        a = base * (k + 1) + 0.1 * torch.randn(N, N, generator=g, dtype=torch.float64)
        b = a + 0.01 * torch.randn(N, N, generator=g, dtype=torch.float64)
        setattr(f1, n, a.cuda())
        setattr(f2, n, b.cuda())
    return f1, f2


def _params(P, seed):
    p = P.init_params(seed, scale_last=1.0)
    rng = np.random.default_rng(seed + 7)
    o = 0
    for ci, co in P.LAYERS:
        o += 9 * ci * co
        p[o:o + co] = rng.normal(0, 0.1, co)
        o += co
    return p


def _bf16_bits_to_f64(t):
    return (t.to(torch.int32) << 16).view(torch.float32).double()


@pytest.fixture(scope='module')
def net41(P):
    N = 41
    params = _params(P, 1)
    pr = P.FieldPredictor(N, params=params)
    f1, f2 = _fields(N, 3)
    pr.pack(f1, f2)
    pr.forward()
    pr.check_errors()
    x = _bf16_bits_to_f64(pr.buffer('input')).view(N, N + 1, 32).cpu().numpy()
    y = pr.buffer('output').view(N, N + 1, 16).double().cpu().numpy()
    return types.SimpleNamespace(N=N, params=params, pr=pr, f1=f1, f2=f2, x=x, y=y)


def test_pack_matches_oracle(P, net41):
    N = net41.N
    f1 = [getattr(net41.f1, n).cpu().numpy() for n in P.FIELDS_IN]
    f2 = [getattr(net41.f2, n).cpu().numpy() for n in P.FIELDS_IN]
    s_in, _ = PO.scales(f1, f2)
    want = PO.bf16(PO.pack(f1, f2, s_in)).astype(np.float64)
    assert np.array_equal(net41.x[:, :N], want)
    assert np.all(net41.x[:, N] == 0)          # the pad column


def test_forward_matches_oracle(P, net41):
    N = net41.N
    want, _ = PO.forward(net41.params, net41.x[:, :N])
    got = net41.y[:, :N]
    d = got[..., :5] - want[..., :5]
    assert np.abs(d).max() <= FWD_MAX_TOL * np.abs(want[..., :5]).max()
    assert np.sqrt((d ** 2).mean()) <= FWD_RMS_TOL * np.sqrt((want[..., :5] ** 2).mean())
    assert np.all(net41.y[:, N] == 0)


def test_gradients_match_oracle(P, net41):
    N, pr = net41.N, net41.pr
    tgt = np.zeros((N, N + 1, 16), np.float32)
    tgt[:, :N, :5] = np.random.default_rng(9).normal(size=(N, N, 5))
    pr.buffer('target').copy_(torch.from_numpy(tgt.ravel()).cuda())
    pr.loss.zero_()
    pr.backward()
    pr.check_errors()
    got = pr.grad().double().cpu().numpy()
    loss, want, _ = PO.loss_and_grad(net41.params, net41.x[:, :N], tgt[:, :N].astype(np.float64))
    assert abs(float(pr.loss.item()) - loss) <= 1e-4 * loss
    o = 0
    for k, (ci, co) in enumerate(P.LAYERS):
        for sl in (slice(o, o + 9 * ci * co), slice(o + 9 * ci * co, o + 9 * ci * co + co)):
            assert np.linalg.norm(got[sl] - want[sl]) <= GRAD_TOL * np.linalg.norm(want[sl]), (k, sl)
        o += 9 * ci * co + co


def test_adam_step_moves_against_gradient(P, net41):
    pr = net41.pr
    before = pr.params().double().cpu().numpy()
    g = pr.grad().double().cpu().numpy()
    pr.adam(1e-3)
    after = pr.params().double().cpu().numpy()
    moved = after - before
    big = np.abs(g) > 1e-3 * np.abs(g).max()
    # the first Adam step is -lr * sign(g) (bias-corrected m / sqrt(v))
    assert np.allclose(moved[big], -1e-3 * np.sign(g[big]), rtol=1e-3, atol=1e-6)
    pr.set_params(net41.params)


@pytest.fixture(scope='module')
def sim161(P):
    cfg = make_config(161, 0.05, 0.05, 300, amplitude=0.05)
    sim = P.Stepper(cfg, (0.05, 1.0, 1.0))
    for _ in range(20):
        sim.step_plain()
    return sim


def _snapshot(sim):
    return ([{n: getattr(b, n).clone() for n in STATE} for b in sim.bufs], sim.prev, sim.cur, sim.xi)


def _restore(sim, snap):
    bufs, sim.prev, sim.cur, sim.xi = snap
    for b, s in zip(sim.bufs, bufs):
        for n in STATE:
            getattr(b, n).copy_(s[n])


def test_first_pass_and_exact_prediction_reproduce_plain_step(P, sim161):
    import ctypes
    from lcode3d_b200 import _lib
    sim = sim161
    snap = _snapshot(sim)
    sim.step_plain()
    plain = {n: getattr(sim.state, n).clone() for n in STATE}
    _restore(sim, snap)
    sim.step_plain(record_first=True)
    rec = {n: getattr(sim.state, n).clone() for n in STATE}
    F1 = {n: sim.first[n].clone() for n in P.FIELDS_6}
    for n in STATE:
        assert torch.equal(rec[n], plain[n]), n
    _restore(sim, snap)
    for n in P.FIELDS_6:
        sim.pred[n].copy_(F1[n])
    o = sim._out()
    sim._beam()
    preds = (ctypes.c_void_p * 6)(*[sim.pred[n].data_ptr() for n in P.FIELDS_6])
    _lib.check(_lib.lib.lc3d_step_arrays_predicted(
        sim.solver.ctx, ctypes.byref(P._sp(sim.state)), ctypes.byref(P._sp(sim.bufs[o])),
        ctypes.c_void_p(sim.beam.data_ptr()), preds, ctypes.c_void_p(sim.residual.data_ptr()),
        P.L._stream()), 'predicted step')
    sim._advance(o)
    for n in STATE:
        assert torch.equal(getattr(sim.state, n), plain[n]), n
    num = max(float((plain[n] - F1[n]).abs().max()) for n in P.FIELDS_OUT)
    den = max(float(plain[n].abs().max()) for n in P.FIELDS_OUT)
    assert float(sim.residual.item()) == pytest.approx(num / den, rel=1e-12)
    # lc3d_fields_rel_diff of the same pair
    a = (ctypes.c_void_p * 6)(*[F1[n].data_ptr() for n in P.FIELDS_6])
    b = (ctypes.c_void_p * 6)(*[plain[n].data_ptr() for n in P.FIELDS_6])
    _lib.check(_lib.lib.lc3d_fields_rel_diff(sim.solver.ctx, a, b, ctypes.c_void_p(sim.error.data_ptr()),
                                             P.L._stream()), 'rel diff')
    assert float(sim.error.item()) == pytest.approx(num / den, rel=1e-12)
    _restore(sim, snap)


def _cfg_scan(N=161, steps=400):
    def mk(beam):
        return make_config(N, 16.0 / (N - 1), 0.01, steps, amplitude=beam[0], sigma_r=beam[1])
    return mk


def test_training_beats_linear_extrapolation(P):
    """The network trained on three solver runs predicts the first-pass
    correction of a held-out run better than linear extrapolation (zero
    output): this is what the predictor gains over the method without it."""
    mk = _cfg_scan()
    pr = P.FieldPredictor(161, seed=0)
    hist = P.train_streaming(pr, mk, [(0.05, 0.9, 1.0), (0.3, 1.2, 1.0), (0.15, 1.0, 1.0)], 400, every=4,
                             epochs_per_run=6, lr=2e-3, lr_final=2e-4)
    assert hist[-1] < hist[0]
    held = (0.1, 1.1, 1.0)
    smp, _ = P.generate_samples(pr, mk(held), held, 400, every=9, start=20)
    net, base = P.evaluate(pr, smp)
    assert net < 0.5 * base, (net, base)


def test_run_learned_policy(P):
    mk = _cfg_scan(steps=120)
    beam = (0.2, 1.0, 1.0)
    pr = P.FieldPredictor(161, seed=0)
    ez_plain, st0, _ = P.run_learned(mk(beam), beam, 120, pr, tol=-1.0)
    assert st0['learned_steps'] == 0 and st0['fallback_rate'] == 1.0
    assert st0['plain_steps'] + st0['verify_steps'] == 120
    ez_l, st1, _ = P.run_learned(mk(beam), beam, 120, pr, tol=float('inf'), verify_every=5)
    assert st1['learned_steps'] + st1['plain_steps'] + st1['verify_steps'] == 120
    assert st1['learned_steps'] == 120 - 20 - st1['verify_steps'] and st1['fallback_rate'] == 0.0
    # plain steps agree with the golden-free reference loop (the same state buffers, plain method)
    sim = P.Stepper(mk(beam), beam)
    ez = []
    for _ in range(120):
        sim.step_plain()
        ez.append(float(sim.state.Ez[80, 80]))
    assert np.array_equal(ez_plain, np.array(ez))
    # the first 20 steps of the learned run are plain
    assert np.array_equal(ez_l[:20], ez_plain[:20])
