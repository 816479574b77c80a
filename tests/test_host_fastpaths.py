"""lcode.solver_for: the cached solver is found from the raw config values;
a changed attribute selects (or makes) another solver. Host logic only: the
Solver and the device queries are stood in for."""
import pytest
import torch

from lcode3d_b200 import lcode
from make_golden import make_config


@pytest.fixture
def fake(monkeypatch):
    made = []

    class FakeSolver:
        def __init__(self, params, device):
            made.append((params.grid_steps, params.precision, device))

    monkeypatch.setattr(lcode, 'Solver', FakeSolver)
    monkeypatch.setattr(lcode, '_cuda_seen', True)
    monkeypatch.setattr(lcode.torch.cuda, 'current_device', lambda: 0)
    monkeypatch.setattr(lcode, '_device', lambda: torch.device('cuda', 0))
    monkeypatch.setattr(lcode, '_solvers', {})
    monkeypatch.setattr(lcode, '_solvers_raw', {})
    return made


def test_same_config_same_solver(fake):
    cfg = make_config(41, 0.1, 0.05, 10, amplitude=0.3)
    s1 = lcode.solver_for(cfg)
    s2 = lcode.solver_for(cfg)
    assert s1 is s2 and len(fake) == 1


def test_changed_attribute_changes_solver(fake):
    cfg = make_config(41, 0.1, 0.05, 10, amplitude=0.3)
    s64 = lcode.solver_for(cfg)
    cfg.lc3d_precision = 'fft32'
    s32 = lcode.solver_for(cfg)
    assert s32 is not s64 and len(fake) == 2
    cfg.lc3d_precision = 'fp64'
    assert lcode.solver_for(cfg) is s64 and len(fake) == 2
    cfg.grid_steps = 61
    assert lcode.solver_for(cfg) is not s64 and len(fake) == 3


def test_equal_configs_share_a_solver(fake):
    a = make_config(41, 0.1, 0.05, 10, amplitude=0.3)
    b = make_config(41, 0.1, 0.05, 10, amplitude=0.3)
    assert lcode.solver_for(a) is lcode.solver_for(b) and len(fake) == 1


def test_const_copy_skipped_only_for_unwritten_same_arrays():
    # Solver.set_const / set_virt copy again after an in-place write (a
    # GPUArraysView assignment, t.copy_, t[...] = ...), not only after the
    # arrays are replaced
    a, b = torch.zeros(4, dtype=torch.float64), torch.ones(4, dtype=torch.float64)
    seen = lcode.Solver._seen((a, b))
    assert lcode.Solver._unchanged((a, b), seen)
    assert not lcode.Solver._unchanged((a, b.clone()), seen)
    b[1] = 5.0
    assert not lcode.Solver._unchanged((a, b), seen)
    seen = lcode.Solver._seen((a, b))
    a.view(2, 2)[0].copy_(torch.ones(2, dtype=torch.float64))   # a write through a view
    assert not lcode.Solver._unchanged((a, b), seen)
    assert not lcode.Solver._unchanged((a, b), None)
