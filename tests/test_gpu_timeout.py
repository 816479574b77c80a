"""Failure detection on the GPU: a bounded wait that runs out.

Every wait in the tensor-core pipeline of the mixed-precision transforms is
bounded. lc3d_test_wait_limit shortens the bound and makes the pipeline's
producer issue no loads, so the consumer's wait for its first stage runs out
with nothing in flight. The kernel must then give up, free its tensor memory,
raise the timeout flag and return, and the context must stay usable: the
next call is normal and reproduces the earlier result bit for bit. Nothing
here faults, traps or hangs the GPU; the wait that runs out is bounded at
100,000 clock cycles."""
import ctypes
import time

import numpy as np
import pytest

torch = pytest.importorskip('torch')

from make_golden import make_config  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def L():
    if not torch.cuda.is_available():
        pytest.skip('no GPU')
    import lcode3d_b200 as L
    L.lcode.check_errors = True
    return L


def test_bounded_wait_runs_out_and_context_recovers(L):
    from lcode3d_b200 import _lib
    lib = _lib.lib
    N = 41
    cfg = make_config(N, 0.1, 0.05, 10, amplitude=0.3)
    cfg.lc3d_precision = 'mixed'
    cfg.lc3d_mixed_slices = 4
    rng = np.random.default_rng(7)
    jx = torch.from_numpy(rng.normal(size=(N, N))).cuda()
    jy = torch.from_numpy(rng.normal(size=(N, N))).cuda()
    s = L.solver_for(cfg)
    ref = L.calculate_Ez(cfg, jx, jy).clone()          # a normal call (flag checked)
    torch.cuda.synchronize()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    out = torch.empty_like(ref)
    _lib.check(lib.lc3d_test_wait_limit(s.ctx, 100000, 1), 'lc3d_test_wait_limit')
    try:
        t0 = time.perf_counter()
        _lib.check(lib.lc3d_calculate_Ez(s.ctx, ctypes.c_void_p(jx.data_ptr()), ctypes.c_void_p(jy.data_ptr()),
                                         ctypes.c_void_p(out.data_ptr()), stream), 'lc3d_calculate_Ez')
        rc = lib.lc3d_check_error(s.ctx, stream)
        dt = time.perf_counter() - t0
    finally:
        _lib.check(lib.lc3d_test_wait_limit(s.ctx, 0, 0), 'lc3d_test_wait_limit')
    print(f'timed-out call returned {_lib.strerror(rc)!r} after {dt * 1e3:.1f} ms')
    assert rc == _lib.ERR_TIMEOUT
    assert dt < 5.0
    assert lib.lc3d_check_error(s.ctx, stream) == _lib.OK   # the flag was cleared by the read
    again = L.calculate_Ez(cfg, jx, jy)                    # same context, default bound
    torch.cuda.synchronize()
    assert torch.equal(again, ref)
