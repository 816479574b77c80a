"""bench.py's reference arm on the host cores (no GPU): one JSON line with
the contract's keys on rank 0, nothing on the other ranks of a torchrun
launch."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(extra_env=None):
    env = dict(os.environ)
    env.update(extra_env or {})
    return subprocess.run([sys.executable, os.path.join(ROOT, 'bench.py'), '--impl', 'reference', '--grid', '161',
                           '--pre', '2', '--steps', '2', '--warmup', '1'],
                          cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_line():
    r = run_bench()
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith('{')]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d['impl'] == 'reference'
    for k in ('metric', 'value', 'unit', 'steps', 'warmup', 'ms_per_step', 'higher_is_better', 'config',
              'cpu_baseline', 'e2e'):
        assert k in d, k
    assert d['value'] > 0 and d['higher_is_better'] is True
    assert d['steps'] == 2 and d['warmup'] == 1
    assert d['config']['grid_steps'] == 161 and d['config']['start_xi_step'] == 2
    cb = d['cpu_baseline']
    assert cb['kind'] == 'port' and cb['cores'] >= 1 and cb['value'] == d['value']
    assert d['e2e'] == {'value': d['value'], 'unit': d['unit'], 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}


def test_reference_arm_other_ranks_print_nothing():
    r = run_bench({'RANK': '1', 'WORLD_SIZE': '2', 'LOCAL_RANK': '1'})
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [l for l in r.stdout.splitlines() if l.startswith('{')]
