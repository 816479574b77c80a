"""The CPU oracle against the reference's own outputs (golden vectors made by
tests/golden/make_golden.py from the reference lcode.py) and against
known answers from mathematics. CPU only."""
import os
import types

import numpy as np
import pytest

from conftest import GOLDEN

from make_golden import beam_array, make_config  # noqa: E402
from oracle import lcode_oracle as O  # noqa: E402

STATE = ('x_offt', 'y_offt', 'px', 'py', 'pz', 'Ex', 'Ey', 'Ez', 'Bx', 'By',
         'Bz', 'ro', 'jx', 'jy', 'jz')


@pytest.fixture(scope='module')
def stages():
    g = np.load(os.path.join(GOLDEN, 'stages_n41.npz'))
    cfg = make_config(int(g['grid_steps']), float(g['grid_step_size']),
                      float(g['xi_step_size']), 10, amplitude=0.3)
    xs, ys, const, virt, _ = O.init(cfg)
    prev = types.SimpleNamespace(**{k[5:]: g[k] for k in g.files if k.startswith('prev_')})
    return g, cfg, const, virt, prev


def test_init_bitwise(stages):
    g, cfg, const, virt, _ = stages
    assert cfg.reflect_boundary == float(g['reflect_boundary'])
    for k in ('m', 'q', 'x_init', 'y_init', 'ro_initial'):
        np.testing.assert_array_equal(getattr(const, k), g['const_' + k])
    for k in ('influence_prev', 'influence_next', 'indices_prev', 'indices_next', 'fine_grid'):
        np.testing.assert_array_equal(getattr(virt, k), g['virt_' + k])


def test_particle_stages_bitwise(stages):
    """Estimate, pusher and deposition reproduce the reference bit for bit
    (the deposition sums in the serial order of the fixture)."""
    g, cfg, c, virt, P = stages
    ex, ey = O.move_estimate_wo_fields(cfg, c.m, c.x_init, c.y_init, P.x_offt, P.y_offt, P.px, P.py, P.pz)
    np.testing.assert_array_equal(ex, g['est_x_offt'])
    np.testing.assert_array_equal(ey, g['est_y_offt'])
    mv = O.move_smart(cfg, c.m, c.q, c.x_init, c.y_init, P.x_offt, P.y_offt, ex, ey,
                      P.px, P.py, P.pz, P.Ex, P.Ey, P.Ez, P.Bx, P.By, P.Bz)
    for k, v in zip(('x_offt', 'y_offt', 'px', 'py', 'pz'), mv):
        np.testing.assert_array_equal(v, g['move_' + k])
    dep = O.deposit(cfg, c.ro_initial, mv[0], mv[1], c.m, c.q, mv[2], mv[3], mv[4], virt)
    for k, v in zip(('ro', 'jx', 'jy', 'jz'), dep):
        np.testing.assert_array_equal(v, g['dep_' + k])


def test_reflection_exercised(stages):
    g, cfg, c, virt, P = stages
    flipped = np.sign(g['move_px']) != np.sign(g['prev_px'])
    assert flipped.sum() > 0
    assert np.abs(c.x_init + g['est_x_offt']).max() <= cfg.reflect_boundary


def test_field_solvers(stages):
    g, cfg, c, virt, P = stages
    ro, jx, jy, jz = (g['dep_' + k] for k in ('ro', 'jx', 'jy', 'jz'))
    F = O.calculate_Ex_Ey_Bx_By(cfg, P.Ex, P.Ey, P.Bx, P.By, g['beam_ro'], ro, jx, jy, jz, P.jx, P.jy)
    for k, v in zip(('Ex', 'Ey', 'Bx', 'By'), F):
        assert O.relative_error(v, g['fld_' + k]) < 1e-14, k
    assert O.relative_error(O.calculate_Ez(cfg, jx, jy), g['fld_Ez']) < 1e-14
    assert O.relative_error(O.calculate_Bz(cfg, jx, jy), g['fld_Bz']) < 1e-14
    cfg0 = make_config(41, 0.1, 0.05, 10, amplitude=0.3)
    cfg0.field_solver_subtraction_trick = 0
    O.init(cfg0)
    F0 = O.calculate_Ex_Ey_Bx_By(cfg0, P.Ex, P.Ey, P.Bx, P.By, g['beam_ro'], ro, jx, jy, jz, P.jx, P.jy)
    for k, v in zip(('Ex', 'Ey', 'Bx', 'By'), F0):
        assert O.relative_error(v, g['fld0_' + k]) < 1e-14, k


@pytest.mark.parametrize('variant_A', [True, False])
def test_step(stages, variant_A):
    g, cfg, c, virt, P = stages
    cfg = make_config(41, 0.1, 0.05, 10, amplitude=0.3)
    cfg.field_solver_variant_A = variant_A
    O.init(cfg)
    new = O.step(cfg, c, virt, P, g['beam_ro'])
    pre = 'step_' if variant_A else 'stepB_'
    for k in STATE:
        assert O.relative_error(getattr(new, k), g[pre + k]) < 1e-14, k


def _dst1(x):
    n = len(x)
    k = np.arange(1, n + 1)
    return np.array([2 * np.sum(x * np.sin(np.pi * kk * k / (n + 1))) for kk in k])


def _dct1(x):
    n = len(x)
    k = np.arange(n)
    c = np.full(n, 2.0)
    c[0] = c[-1] = 1
    return np.array([np.sum(c * x * np.cos(np.pi * kk * k / (n - 1))) for kk in k])


def test_transforms_known_answers(stages):
    """dst2d = DST-I x DST-I, dct2d = -(DCT-I x DCT-I), mix2d = DST-I(axis 0)
    x DCT-I(axis 1) with zero border rows: against explicit sums and against
    the reference's padded-FFT constructions."""
    g = stages[0]
    rng = np.random.default_rng(1)
    a = rng.normal(size=(7, 7))
    exp = np.apply_along_axis(_dst1, 1, np.apply_along_axis(_dst1, 0, a))
    np.testing.assert_allclose(O.dst2d(a), exp, rtol=0, atol=1e-12)
    b = rng.normal(size=(9, 9))
    exp = -np.apply_along_axis(_dct1, 1, np.apply_along_axis(_dct1, 0, b))
    np.testing.assert_allclose(O.dct2d(b), exp, rtol=0, atol=1e-12)
    cm = rng.normal(size=(5, 7))
    exp = np.apply_along_axis(_dct1, 1, np.apply_along_axis(_dst1, 0, cm))
    out = O.mix2d(cm)
    np.testing.assert_allclose(out[1:-1], exp, rtol=0, atol=1e-12)
    assert not out[0].any() and not out[-1].any()
    assert O.relative_error(O.dst2d(g['tr_dst_in']), g['tr_dst_out']) < 1e-14
    assert O.relative_error(O.dct2d(g['tr_dct_in']), g['tr_dct_out']) < 1e-14
    assert O.relative_error(O.mix2d(g['tr_mix_in']), g['tr_mix_out']) < 1e-14


def test_poisson_manufactured():
    """The Dirichlet solve inverts the 5-point Laplacian: for
    Ez = sin(pi x/Lx) sin(pi y/Ly) sampled on the grid, feeding back the
    discrete Laplacian returns Ez (eigenvalues lam_k of lcode.py:152-154)."""
    cfg = make_config(21, 0.1, 0.05, 1, amplitude=0)
    N, h = 21, 0.1
    rng = np.random.default_rng(3)
    u = np.zeros((N, N))
    u[1:-1, 1:-1] = rng.normal(size=(N - 2, N - 2))
    lap = np.zeros_like(u)
    lap[1:-1, 1:-1] = (u[2:, 1:-1] + u[:-2, 1:-1] + u[1:-1, 2:] + u[1:-1, :-2] - 4 * u[1:-1, 1:-1]) / h ** 2
    f = O.dst2d(-lap[1:-1, 1:-1]) * O.dirichlet_matrix(N, h)
    np.testing.assert_allclose(O.dst2d(f), u[1:-1, 1:-1], rtol=0, atol=1e-12)


def test_tsc_weights():
    x = np.linspace(-0.77, 0.91, 101)
    y = np.linspace(0.33, -0.52, 101)
    i, j, w = O.weights(x, y, 41, 0.1)
    np.testing.assert_allclose(sum(w), 1.0, rtol=0, atol=1e-15)
    # at a cell centre: 0.75^2 in the middle, 0.125 * 0.75 at the edges
    i, j, w = O.weights(np.array([0.25]), np.array([-0.375]), 41, 0.125)
    assert (i[0], j[0]) == (22, 17)
    assert w[4][0] == 0.75 * 0.75 and w[1][0] == 0.75 * 0.125 and w[0][0] == 0.125 * 0.125


def test_charge_neutrality():
    cfg = make_config(41, 0.1, 0.05, 10, amplitude=0.3)
    xs, ys, const, virt, st = O.init(cfg)
    ro, jx, jy, jz = O.deposit(cfg, const.ro_initial, st.x_offt, st.y_offt, const.m, const.q,
                               st.px, st.py, st.pz, virt)
    assert np.abs(ro).max() == 0
    assert np.abs(jx).max() == 0 and np.abs(jz).max() == 0
    assert abs(const.ro_initial.sum() - len(virt.fine_grid) ** 2 * 0.25) < 1e-9


def test_run_n161_head():
    """100 steps of the small production-shaped run (161^2, h=0.05,
    dxi=0.05, A=0.05): on-axis Ez history and field snapshots against the
    reference; the deposition order is the same, the FFTs differ."""
    g = np.load(os.path.join(GOLDEN, 'run_n161.npz'))
    cfg = make_config(161, 0.05, 0.05, 300, amplitude=0.05)
    xs, ys, const, virt, st = O.init(cfg)
    ez = []
    for i in range(100):
        st = O.step(cfg, const, virt, st, beam_array(cfg, i, xs, ys))
        ez.append(st.Ez[80, 80])
        if i == 0:
            for k in ('Ex', 'Ey', 'Ez', 'Bz', 'ro', 'jz'):
                assert O.relative_error(getattr(st, k), g['s1_' + k]) < 1e-13, k
    assert O.relative_error(np.array(ez), g['Ez00'][:100]) < 1e-13
    for k in ('Ex', 'Ey', 'Ez', 'Bz', 'ro', 'jz'):
        assert O.relative_error(getattr(st, k), g['s100_' + k]) < 1e-12, k


def test_run_n641_two_steps():
    """The production grid (641^2, h=0.025, dxi=0.005, A=0.5): two steps
    against the reference's axis/diagonal rows and global sums."""
    g = np.load(os.path.join(GOLDEN, 'run_n641_head.npz'))
    if 's2_axis_Ez' not in g.files:
        pytest.skip('fixture without the step-2 checkpoint')
    cfg = make_config(641, 0.025, 0.005, 3000, amplitude=0.5)
    xs, ys, const, virt, st = O.init(cfg)
    assert abs(const.ro_initial.sum() - float(g['ro_initial_sum'])) < 1e-9
    for i in range(2):
        st = O.step(cfg, const, virt, st, beam_array(cfg, i, xs, ys))
    for k in STATE[5:]:
        a = getattr(st, k)
        scale = float(g['s2_maxabs_' + k])
        assert np.abs(a[320] - g['s2_axis_' + k]).max() <= 1e-12 * scale, k
        assert np.abs(np.diagonal(a) - g['s2_diag_' + k]).max() <= 1e-12 * scale, k


def test_golden_floor_of_two_orders(tmp_path):
    """make_golden's order-sensitivity floor: for each recorded quantity the
    largest serial-vs-reversed difference relative to the serial values'
    largest modulus, written beside the serial values."""
    import make_golden as M
    ser = {'Ez00': np.array([1.0, -2.0, 4.0]), 's500_axis_ro': np.array([0.5, 0.25]),
           'steps': np.array(3000), 'snapshots': np.array([500])}
    rev = {'Ez00': np.array([1.0, -2.0 + 4e-12, 4.0]), 's500_axis_ro': np.array([0.5, 0.25])}
    a, b = tmp_path / 'ser.npz', tmp_path / 'rev.npz'
    np.savez(a, **ser)
    np.savez(b, **rev)
    M.gen_cfg2_floor(str(a), str(b), str(a))
    g = np.load(a)
    assert abs(float(g['floor_Ez00']) - 1e-12) < 1e-15
    assert g['floor_s500_axis_ro'] == 0.0
    assert 'floor_steps' not in g.files and 'floor_snapshots' not in g.files
    assert np.array_equal(g['Ez00'], ser['Ez00'])
