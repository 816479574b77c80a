"""CPU oracle of the learned field predictor (test infrastructure only).

A numpy restatement of the network that lcode3d_b200/csrc/predictor.cu runs
on the GPU, forward and backward, used by the tests to check the CUDA
kernels' outputs and gradients. It is the checker, never the product: only
tests/ and __graft_entry__.smoke() import it.

The predictor has no counterpart in the reference (lotov/lcode3d). It
replaces the first particle pass of the reference's step (lcode.py:846-871),
whose fields it is trained to predict; the pass it stands in for is the
oracle of its training data, and the reference's corrector (lcode.py:
876-901) judges it at run time.

Network (images [H][W][C], zero padding, 3x3 cross-correlations with weights
W[tap][Cout][Cin], tap = 3 (dy + 1) + (dx + 1), out[y][x] = sum_tap
in[y + dy][x + dx] W[tap]^T + b):
    e1 = relu(conv1(x0));   e2 = relu(conv2(pool(e1)));  e3 = relu(conv3(pool(e2)))
    u3 = conv4(e3);         d2 = relu(up(u3) + e2);      u2 = conv5(d2)
    d1 = relu(up(u2) + e1); y = conv6(d1)
pool: 2x2 average over the valid children (ceil mode); up: nearest
neighbour. With ``use_bf16=True`` every stored activation is rounded to bf16 at
the points where the GPU stores bf16 (inputs, weights, all activations but
y), the arithmetic itself stays float64; with ``use_bf16=False`` the network is
pure float64, which the finite-difference self-check uses.
"""
import numpy as np

LAYERS = ((32, 32), (32, 64), (64, 128), (128, 64), (64, 32), (32, 16))   # (Cin, Cout)
N_IN, N_OUT = 27, 5


def num_params():
    return sum(9 * co * ci + co for ci, co in LAYERS)


def bf16(x):
    """Round float32 values to bfloat16 (nearest, ties to even), as float32."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32)).view(np.uint32).astype(np.uint64)
    r = ((a + 0x7FFF + ((a >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def unflatten(params):
    """[(W [9][Cout][Cin], b [Cout])] from the flat float32 parameter array
    (per layer: weights, then biases)."""
    out, o = [], 0
    for ci, co in LAYERS:
        w = np.asarray(params[o:o + 9 * co * ci], np.float64).reshape(9, co, ci)
        o += 9 * co * ci
        b = np.asarray(params[o:o + co], np.float64)
        o += co
        out.append((w, b))
    return out


def _shift(x, dy, dx):
    """s[y][x] = x[y + dy][x + dx] with zeros outside."""
    H, W = x.shape[:2]
    p = np.pad(x, ((1, 1), (1, 1), (0, 0)))
    return p[1 + dy:1 + dy + H, 1 + dx:1 + dx + W]


def conv(x, w, b):
    y = np.zeros(x.shape[:2] + (w.shape[1],))
    for tap in range(9):
        y += _shift(x, tap // 3 - 1, tap % 3 - 1) @ w[tap].T
    return y + b


def conv_bwd(x, w, g, g_bf=None):
    """(dL/dx, dL/dW, dL/db) of y = conv(x, w, b) given g = dL/dy. dL/dx and
    dL/dW are computed from ``g_bf`` when it is given: the GPU's backward
    data and weight passes run on the tensor cores and read g rounded to
    bf16; the bias gradient uses g as it is."""
    gd = g if g_bf is None else g_bf
    dw = np.zeros_like(w)
    dx = np.zeros(x.shape)
    for tap in range(9):
        dy_, dx_ = tap // 3 - 1, tap % 3 - 1
        dw[tap] = np.einsum('hwo,hwi->oi', gd, _shift(x, dy_, dx_))
        dx += _shift(gd, -dy_, -dx_) @ w[tap]
    return dx, dw, g.sum(axis=(0, 1))


def pool(x):
    H, W, C = x.shape
    Ho, Wo = (H + 1) // 2, (W + 1) // 2
    s = np.zeros((Ho, Wo, C))
    n = np.zeros((Ho, Wo, 1))
    for dy in range(2):
        for dx in range(2):
            part = x[dy::2, dx::2]
            s[:part.shape[0], :part.shape[1]] += part
            n[:part.shape[0], :part.shape[1]] += 1
    return s / n, n


def pool_bwd(g, n, shape):
    H, W = shape[:2]
    up = np.repeat(np.repeat(g / n, 2, axis=0), 2, axis=1)
    return up[:H, :W]


def up(u, shape):
    return np.repeat(np.repeat(u, 2, axis=0), 2, axis=1)[:shape[0], :shape[1]]


def up_bwd(g, shape):
    Ho, Wo = shape[:2]
    s = np.zeros((Ho, Wo, g.shape[2]))
    for dy in range(2):
        for dx in range(2):
            part = g[dy::2, dx::2]
            s[:part.shape[0], :part.shape[1]] += part
    return s


def relu(x):
    return np.maximum(x, 0.0)


def forward(params, x0, use_bf16=True):
    """Forward pass; x0 is [H][W][32] (channels >= 18 zero). Returns (y, cache)."""
    R = (lambda a: bf16(a).astype(np.float64)) if use_bf16 else (lambda a: np.asarray(a, np.float64))
    L = [(R(w), np.asarray(b, np.float64)) for w, b in unflatten(params)]
    c = {'x0': R(x0), 'L': L}
    c['e1'] = R(relu(conv(c['x0'], *L[0])))
    p1, c['n1'] = pool(c['e1'])
    c['p1'] = R(p1)
    c['e2'] = R(relu(conv(c['p1'], *L[1])))
    p2, c['n2'] = pool(c['e2'])
    c['p2'] = R(p2)
    c['e3'] = R(relu(conv(c['p2'], *L[2])))
    c['u3'] = R(conv(c['e3'], *L[3]))
    c['d2'] = R(relu(up(c['u3'], c['e2'].shape) + c['e2']))
    c['u2'] = R(conv(c['d2'], *L[4]))
    c['d1'] = R(relu(up(c['u2'], c['e1'].shape) + c['e1']))
    y = conv(c['d1'], *L[5])
    if use_bf16:
        y = y.astype(np.float32).astype(np.float64)
    return y, c


def loss_and_grad(params, x0, target, use_bf16=True):
    """MSE over the 5 used output channels and the flat gradient of all
    parameters (the layout of ``params``)."""
    y, c = forward(params, x0, use_bf16)
    H, W = x0.shape[:2]
    d = np.zeros_like(y)
    d[..., :N_OUT] = y[..., :N_OUT] - target[..., :N_OUT]
    loss = float((d ** 2).sum() / (N_OUT * H * W))
    g = 2.0 * d / (N_OUT * H * W)
    L = c['L']
    # the output gradients the backward data and weight passes read: bf16 on the GPU
    RG = (lambda a: bf16(a).astype(np.float64)) if use_bf16 else (lambda a: a)
    grads = [None] * 6
    # conv6
    gd1, *grads[5] = conv_bwd(c['d1'], L[5][0], g, RG(g))
    gd1 = gd1 * (c['d1'] > 0)
    gu2 = up_bwd(gd1, c['u2'].shape)
    # conv5
    gd2, *grads[4] = conv_bwd(c['d2'], L[4][0], gu2, RG(gu2))
    gd2 = gd2 * (c['d2'] > 0)
    gu3 = up_bwd(gd2, c['u3'].shape)
    # conv4
    ge3, *grads[3] = conv_bwd(c['e3'], L[3][0], gu3, RG(gu3))
    ge3 = ge3 * (c['e3'] > 0)
    # conv3
    gp2, *grads[2] = conv_bwd(c['p2'], L[2][0], ge3, RG(ge3))
    ge2 = (gd2 + pool_bwd(gp2, c['n2'], c['e2'].shape)) * (c['e2'] > 0)
    # conv2
    gp1, *grads[1] = conv_bwd(c['p1'], L[1][0], ge2, RG(ge2))
    ge1 = (gd1 + pool_bwd(gp1, c['n1'], c['e1'].shape)) * (c['e1'] > 0)
    # conv1
    _, *grads[0] = conv_bwd(c['x0'], L[0][0], ge1, RG(ge1))
    flat = np.concatenate([np.concatenate([dw.ravel(), db.ravel()]) for dw, db in grads])
    return loss, flat, y


def scales(f1, f2, in_mult=None, out_mult=None):
    """Per-sample channel scales as the GPU computes them: root mean squares
    of the 9 fields of t-1 and of their differences to t-2 over the grid
    (times the multipliers; 1 where a mean square is 0), and the output
    scale: the root mean square of the differences of Ex, Ey, Bx, By, Bz
    (channels 13..17)."""
    in_mult = np.ones(18) if in_mult is None else np.asarray(in_mult, float)
    out_mult = np.ones(5) if out_mult is None else np.asarray(out_mult, float)
    rms = np.array([np.sqrt(np.mean(f1[c] ** 2)) for c in range(9)] +
                   [np.sqrt(np.mean((f1[c] - f2[c]) ** 2)) for c in range(9)])
    s_in = np.where(rms > 0, in_mult * rms, 1.0)
    o = np.sqrt(np.mean(rms[13:18] ** 2))
    s_out = np.where(o > 0, out_mult * o, 1.0) * np.ones(5)
    return s_in, s_out


def pack(f1, f2, s_in):
    """Network input [N][N][32] from the 9 fields (ro, jx, jy, jz, Ex, Ey,
    Bx, By, Bz; N x N float64) of t-1 and t-2, before bf16 rounding:
    normalised fields, normalised differences, log10 of the field scales / 4."""
    N = f1[0].shape[0]
    x = np.zeros((N, N, 32), np.float32)
    for c in range(9):
        x[..., c] = (f1[c] * (1.0 / s_in[c])).astype(np.float32)
        x[..., 9 + c] = ((f1[c] - f2[c]) * (1.0 / s_in[9 + c])).astype(np.float32)
        x[..., 18 + c] = np.float32(np.log10(s_in[c]) * 0.25)
    return x
