"""The deposition entry point that allocates nothing, against the usual one.

lc3d_deposit_noalloc is for callers that cannot allocate device memory at
the point where they deposit -- a host program that reserved the GPU's
memory for its own pool and forbids further cudaMalloc, or code that must
not call cudaMalloc (it synchronises the device, and it is not allowed
while a CUDA graph is being captured). It needs no context and keeps its
scratch in a statically sized device array shared by all calls, so this
test makes two calls in a row with different inputs: the second must not
see anything the first left behind.

This file is named to be collected last: if it fails, a run that stops at
the first failure has already run every other test."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip('torch')

from make_golden import make_config  # noqa: E402
from oracle import lcode_oracle as O  # noqa: E402

pytestmark = pytest.mark.gpu

TOL = 1e-13   # the deposition tolerance of the parity tests


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def test_deposit_noalloc_matches_context_deposit():
    if not torch.cuda.is_available():
        pytest.skip('no GPU')
    import lcode3d_b200 as L
    from lcode3d_b200 import _lib

    cfg = make_config(161, 0.05, 0.05, 10, amplitude=0.05)
    xs, ys, const, virt, st = L.init(cfg)
    params = L.lcode.params_of(cfg)
    ip32 = virt.indices_prev.to(torch.int32).contiguous()
    in32 = virt.indices_next.to(torch.int32).contiguous()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(2024)
    x0 = const.x_init.cpu().numpy()
    y0 = const.y_init.cpu().numpy()
    rb = cfg.reflect_boundary * 0.97
    for call, amp in enumerate((0.3, 1.2)):
        x = np.clip(x0 + rng.normal(0, amp, x0.shape), -rb, rb)
        y = np.clip(y0 + rng.normal(0, amp, y0.shape), -rb, rb)
        t = [torch.from_numpy(a).cuda() for a in (x - x0, y - y0, rng.normal(0, 0.3, x0.shape),
                                                    rng.normal(0, 0.3, x0.shape),
                                                    rng.normal(0, 0.3, x0.shape))]
        ref = L.deposit(cfg, const.ro_initial, t[0], t[1], const.m, const.q, t[2], t[3], t[4], virt)
        out = [torch.full_like(ref[0], float('nan')) for _ in range(4)]
        rc = _lib.lib.lc3d_deposit_noalloc(
            ctypes.byref(params), _p(const.ro_initial), _p(t[0]), _p(t[1]), _p(const.m), _p(const.q),
            _p(t[2]), _p(t[3]), _p(t[4]), _p(virt.influence_prev), _p(virt.influence_next), _p(ip32),
            _p(in32), _p(virt.fine_grid), *[_p(o) for o in out], stream)
        assert rc == _lib.OK, _lib.strerror(rc)
        torch.cuda.synchronize()
        for name, a, b in zip(('ro', 'jx', 'jy', 'jz'), out, ref):
            e = O.relative_error(a.cpu().numpy(), b.cpu().numpy())
            assert e <= TOL, (call, name, e)

    # a grid above the static maximum is refused before any device work
    big = make_config(641, 0.025, 0.005, 10, amplitude=0.5)
    rc = _lib.lib.lc3d_deposit_noalloc(
        ctypes.byref(L.lcode.params_of(big)), None, *[_p(t[0])] * 7, *[_p(virt.fine_grid)] * 5,
        *[_p(o) for o in out], stream)
    assert rc == _lib.ERR_SIZE
