"""CPU checks of the learned-predictor oracle and host logic: the numpy
network's backward pass against finite differences (pure float64), its
bf16 rounding against torch's, its parameter layout against liblc3d's and
the product's initialisation (no GPU needed)."""
import numpy as np
import pytest
import torch

from oracle import predictor_oracle as PO


def _tiny_input(H, seed):
    rng = np.random.default_rng(seed)
    x = np.zeros((H, H, 32))
    x[..., :PO.N_IN] = rng.normal(size=(H, H, PO.N_IN))
    t = np.zeros((H, H, 16))
    t[..., :PO.N_OUT] = rng.normal(size=(H, H, PO.N_OUT))
    return x, t


def _params(seed):
    from lcode3d_b200.predictor import init_params
    p = init_params(seed, scale_last=1.0).astype(np.float64)
    rng = np.random.default_rng(seed + 100)
    # non-zero biases so that every bias gradient path is exercised
    o = 0
    for ci, co in PO.LAYERS:
        o += 9 * co * ci
        p[o:o + co] = rng.normal(0, 0.1, co)
        o += co
    return p


def test_num_params_matches_library():
    from lcode3d_b200._lib import lib
    assert PO.num_params() == lib.lc3d_predictor_num_params() == 198480


def test_init_params_layout():
    from lcode3d_b200.predictor import init_params
    p = init_params(3)
    assert p.dtype == np.float32 and p.size == PO.num_params()
    layers = PO.unflatten(p)
    assert np.all(layers[0][0][:, :, PO.N_IN:] == 0)          # padded inputs of conv1
    assert np.all(layers[-1][0][:, PO.N_OUT:, :] == 0)        # unused outputs of conv6
    assert all(np.all(b == 0) for _, b in layers)
    assert np.array_equal(p, init_params(3)) and not np.array_equal(p, init_params(4))


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.normal(size=10000), rng.normal(size=1000) * 1e-30, [0.0, -0.0, 1.0, 65504.0, 3e38]])
    x = x.astype(np.float32)
    want = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(PO.bf16(x), want)


@pytest.mark.parametrize('H', [7, 10])
def test_backward_matches_finite_differences(H):
    """Odd and even sizes (ceil pooling on 7 -> 4 -> 2, 10 -> 5 -> 3)."""
    p = _params(1)
    x, t = _tiny_input(H, 2)
    loss, g, _ = PO.loss_and_grad(p, x, t, use_bf16=False)
    rng = np.random.default_rng(5)
    offs = np.cumsum([0] + [9 * co * ci + co for ci, co in PO.LAYERS])
    idx = []
    for k, (ci, co) in enumerate(PO.LAYERS):
        ci_used = PO.N_IN if k == 0 else ci
        co_used = PO.N_OUT if k == len(PO.LAYERS) - 1 else co
        for _ in range(4):   # weights of used channels
            tap, o_, i_ = rng.integers(9), rng.integers(co_used), rng.integers(ci_used)
            idx.append(offs[k] + (tap * co + o_) * ci + i_)
        idx.append(offs[k] + 9 * co * ci + rng.integers(co_used))   # a bias
    eps = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        fd = (PO.loss_and_grad(pp, x, t, False)[0] - PO.loss_and_grad(pm, x, t, False)[0]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (i, fd, g[i])


def test_scales_and_pack():
    rng = np.random.default_rng(0)
    f1 = [rng.normal(size=(9, 9)) * (c + 1) for c in range(9)]
    f2 = [f + rng.normal(size=(9, 9)) * 1e-3 for f in f1]
    f1[3] = np.zeros((9, 9))
    f2[3] = np.zeros((9, 9))       # an all-zero field: scale 1
    s_in, s_out = PO.scales(f1, f2)
    assert s_in[3] == 1.0 and s_in[12] == 1.0
    assert np.allclose(s_in[0], np.sqrt(np.mean(f1[0] ** 2)))
    assert np.allclose(s_out, np.sqrt(np.mean(s_in[13:18] ** 2)))
    x = PO.pack(f1, f2, s_in)
    assert x.shape == (9, 9, 32) and np.all(x[..., 27:] == 0)
    assert np.allclose(x[..., 18], np.log10(s_in[0]) / 4)
    assert np.allclose(x[..., 0], f1[0] / s_in[0], rtol=1e-6)
    assert np.allclose(np.sqrt(np.mean(x[..., 9].astype(float) ** 2)), 1.0, rtol=1e-5)
