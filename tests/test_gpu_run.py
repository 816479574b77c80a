"""Graph-replayed runs with the device-side beam, checkpoint/resume, and
batches of simulations, against the per-step drop-in path."""
import os

import numpy as np
import pytest

torch = pytest.importorskip('torch')

from make_golden import beam_array, make_config  # noqa: E402
from oracle import lcode_oracle as O  # noqa: E402

pytestmark = pytest.mark.gpu

STATE = ('x_offt', 'y_offt', 'px', 'py', 'pz', 'Ex', 'Ey', 'Ez', 'Bx', 'By', 'Bz', 'ro', 'jx', 'jy', 'jz')


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


def test_run_matches_host_loop(L):
    """lc3d_run (device beam, graph replay, device Ez history) against the
    reference-style host loop of step() with the beam from numpy; the two
    beams differ by rounding of exp/cos only."""
    cfg = make_config(161, 0.05, 0.05, 300, amplitude=0.05)
    xs, ys, const, virt, st0 = L.init(cfg)
    st, ez_host = st0, []
    for i in range(60):
        st = L.step(cfg, const, virt, st, beam_array(cfg, i, xs, ys))
        ez_host.append(float(st.Ez[80, 80]))
    got, ez = L.lcode.run(cfg, const, virt, st0, 0, 60, beam=(0.05, 1.0, 1.0))
    assert rel(ez, np.array(ez_host)) < 1e-12
    for k in STATE:
        assert rel(getattr(got, k), getattr(st, k)) < 1e-11, k
    # the same 60 steps as 25 + 35 (both state parities)
    a, ez_a = L.lcode.run(cfg, const, virt, st0, 0, 25, beam=(0.05, 1.0, 1.0))
    b, ez_b = L.lcode.run(cfg, const, virt, a, 25, 35, beam=(0.05, 1.0, 1.0))
    assert torch.equal(torch.cat([ez_a, ez_b]), ez)
    for k in STATE:
        assert torch.equal(getattr(b, k), getattr(got, k)), k


def test_checkpoint_resume(L, tmp_path):
    cfg = make_config(161, 0.05, 0.05, 300, amplitude=0.05)
    xs, ys, const, virt, st = L.init(cfg)
    for i in range(20):
        st = L.step(cfg, const, virt, st, beam_array(cfg, i, xs, ys))
    path = os.path.join(tmp_path, 'ck.npz')
    L.lcode.save_checkpoint(path, 20, const, virt, st)
    straight = st
    for i in range(20, 30):
        straight = L.step(cfg, const, virt, straight, beam_array(cfg, i, xs, ys))
    xi, c2, v2, s2 = L.lcode.load_checkpoint(path)
    assert xi == 20
    for i in range(20, 30):
        s2 = L.step(cfg, c2, v2, s2, beam_array(cfg, i, xs, ys))
    for k in STATE:
        assert torch.equal(getattr(s2, k), getattr(straight, k)), k


@pytest.mark.parametrize('multi', [False, True])
def test_batch_matches_individual_runs(L, multi):
    """Four simulations of two grid sizes advanced by one graph launch per
    step give bit-identical results to running each on its own, with the
    depositions on each simulation's branch or as one launch over all
    simulations per deposition point."""
    from lcode3d_b200 import batch as B
    specs = [dict(grid_steps=N, grid_step_size=16.0 / (N - 1), xi_step_size=0.01, amplitude=A,
                  sigma_r=sr, length_factor=lf)
             for N, A, sr, lf in ((161, 0.3, 1.0, 1.0), (321, 0.05, 0.7, 1.3), (161, 0.8, 1.5, 0.6),
                                  (321, 0.5, 1.0, 1.0))]
    bt = B.Batch(specs, multi_deposit=multi)
    hist = [h.clone() for h in bt.run(30)]
    hist2 = bt.run(15)
    bt.check_errors()
    for i, spec in enumerate(specs):
        cfg = B.make_config(spec)
        xs, ys, const, virt, st0 = L.init(cfg)
        beam = (spec['amplitude'], spec['sigma_r'], spec['length_factor'])
        st, ez = L.lcode.run(cfg, const, virt, st0, 0, 45, beam=beam)
        assert torch.equal(torch.cat([hist[i], hist2[i]]), ez), i
        final = bt.sims[i].state()
        for k in STATE:
            assert torch.equal(getattr(final, k), getattr(st, k)), (i, k)


def test_autotuner_picks_a_form(L):
    from lcode3d_b200 import batch as B
    choice, timings = B.autotune_transform([161], steps=3)
    assert choice[161] in ('fft', 'dense')
    assert set(timings[161]) == {'fft', 'dense'} and all(v > 0 for v in timings[161].values())


def test_autotuner_picks_tile_shapes(L):
    from lcode3d_b200 import batch as B
    choice, timings = B.autotune([161], steps=2)
    c = choice[161]
    assert c['transform'] in ('fft', 'dense')
    assert c['deposit_rows'] in B.TILE_CHOICES['deposit_rows']
    assert c['fft_ctas_per_sm'] in B.TILE_CHOICES['fft_ctas_per_sm']
    assert len(timings[161]) >= 6 and all(v > 0 for v in timings[161].values())


@pytest.mark.parametrize('tiles', [(4, 0), (8, 2), (16, 1)])
def test_tile_shapes_agree_with_the_oracle(L, tiles):
    """Every deposition tile height and FFT grid cap gives the reference's
    result: 20 steps of the 161^2 run against the oracle (1e-10)."""
    from lcode3d_b200 import _lib
    cfg = make_config(161, 0.05, 0.05, 300, amplitude=0.05)
    cfg.lc3d_fp64_transform = 'fft'   # a context of its own (the default config says 'auto')
    s = L.solver_for(cfg)
    _lib.check(_lib.lib.lc3d_set_tiles(s.ctx, *tiles), 'lc3d_set_tiles')
    try:
        xs, ys, const, virt, st = L.init(cfg)
        ocfg = make_config(161, 0.05, 0.05, 300, amplitude=0.05)
        oxs, oys, oconst, ovirt, ost = O.init(ocfg)
        for i in range(20):
            b = beam_array(cfg, 40 + i, xs, ys)
            st = L.step(cfg, const, virt, st, b)
            ost = O.step(ocfg, oconst, ovirt, ost, b)
        for k in STATE:
            assert rel(getattr(st, k), getattr(ost, k)) < 1e-10, k
    finally:
        _lib.check(_lib.lib.lc3d_set_tiles(s.ctx, 0, 0), 'lc3d_set_tiles')
    for bad in ((3, 0), (32, 0), (8, -1)):
        assert _lib.lib.lc3d_set_tiles(s.ctx, *bad) == _lib.ERR_PARAM


def test_diag_zn_matches_scipy(L):
    """lc3d_diag_zn against the reference's own zn expression (scipy.ndimage
    gaussian_filter, oracle restatement) on a state from a real run and on
    a noisy field; the running maximum is kept like the reference's."""
    cfg = make_config(161, 0.05, 0.05, 300, amplitude=0.05)
    xs, ys, const, virt, st = L.init(cfg)
    for i in range(40):
        st = L.step(cfg, const, virt, st, beam_array(cfg, i, xs, ys))
    ro = st.ro.cpu().numpy()
    rng = np.random.default_rng(3)
    noisy = ro + 1e-3 * rng.normal(size=ro.shape)
    L.lcode.max_zn = 0.0
    a = L.lcode.diags_ro_zn(cfg, st.ro)
    assert a == pytest.approx(O.diags_ro_zn_value(cfg, ro), rel=1e-12)
    b = L.lcode.diags_ro_zn(cfg, torch.from_numpy(noisy).cuda())
    assert b == pytest.approx(max(a, O.diags_ro_zn_value(cfg, noisy)), rel=1e-12)
    assert L.lcode.diags_ro_zn(cfg, st.ro) == b       # running maximum
    # a 641 grid (sigma = 10 cells, 81 taps)
    cfg6 = make_config(641, 0.025, 0.005, 10, amplitude=0.5)
    L.lcode.max_zn = 0.0
    z = rng.normal(size=(641, 641))
    assert L.lcode.diags_ro_zn(cfg6, torch.from_numpy(z).cuda()) == pytest.approx(
        O.diags_ro_zn_value(cfg6, z), rel=1e-12)


def test_host_beam_step_is_device_beam_step(L):
    """lcode.step with the beam in host memory (copied during the first
    deposition, lc3d_step_arrays_host_beam) gives the same bits as with the
    beam already on the device, for pageable and pinned host arrays."""
    cfg = make_config(161, 0.05, 0.05, 300, amplitude=0.05)
    xs, ys, const, virt, st = L.init(cfg)
    a = b = c = st
    for i in range(12):
        beam = beam_array(cfg, i, xs, ys)
        a = L.step(cfg, const, virt, a, beam)                                   # numpy, pageable
        b = L.step(cfg, const, virt, b, torch.from_numpy(beam).cuda())          # device
        c = L.step(cfg, const, virt, c, torch.from_numpy(beam).pin_memory())    # pinned
    for k in STATE:
        assert torch.equal(getattr(a, k), getattr(b, k)), k
        assert torch.equal(getattr(c, k), getattr(b, k)), k


@pytest.mark.parametrize('N,h,c,f', [(41, 0.1, 3, 2), (61, 0.1, 2, 3), (81, 0.1, 4, 1), (161, 0.05, 3, 2),
                                     (641, 0.025, 3, 2)])
def test_init_on_device_matches_host_init(L, N, h, c, f):
    """lc3d_init_plasma (plasma layout, ion background, initial state built
    on the device) against the host layout of init(): bit-identical."""
    cfg = make_config(N, h, 0.05, 10, amplitude=0.1)
    cfg.plasma_coarseness, cfg.plasma_fineness = c, f
    cfg.reflect_padding_steps = max(cfg.reflect_padding_steps, c + 2)
    xs, ys, const, virt, st = L.init(cfg)
    xs2, ys2, const2, virt2, st2 = L.lcode.init_device(cfg)
    assert np.array_equal(xs, xs2) and np.array_equal(ys, ys2)
    for k in ('m', 'q', 'x_init', 'y_init', 'ro_initial'):
        assert torch.equal(L.lcode._f64(getattr(const, k)), getattr(const2, k)), k
    for k in ('influence_prev', 'influence_next', 'fine_grid'):
        assert torch.equal(L.lcode._f64(getattr(virt, k)), getattr(virt2, k)), k
    for k in ('indices_prev', 'indices_next'):
        assert torch.equal(torch.as_tensor(getattr(virt, k)).cuda().long(), getattr(virt2, k)), k
    for k in STATE:
        assert torch.equal(L.lcode._f64(getattr(st, k)), getattr(st2, k)), k
