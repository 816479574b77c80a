"""build() must work on a fresh checkout: the package loads liblc3d.so on
import, so the build module is loaded on its own (host-only checks)."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_build_module_loads_without_the_package():
    import __graft_entry__ as g
    before = set(sys.modules)
    b = g._load_file('lc3d_build_probe', os.path.join(ROOT, 'lcode3d_b200', 'build.py'))
    assert b.LIB.endswith(os.path.join('lcode3d_b200', 'liblc3d.so'))
    assert all(os.path.exists(s) for s in b.sources())
    # loading the build module imported nothing of the package itself
    new = set(sys.modules) - before
    assert not any(m == 'lcode3d_b200' or m.startswith('lcode3d_b200.') for m in new)


def test_build_sources_cover_every_cuda_file():
    import __graft_entry__ as g
    b = g._load_file('lc3d_build_probe2', os.path.join(ROOT, 'lcode3d_b200', 'build.py'))
    csrc = os.path.join(ROOT, 'lcode3d_b200', 'csrc')
    on_disk = sorted(f for f in os.listdir(csrc) if f.endswith('.cu'))
    assert sorted(os.path.basename(s) for s in b.sources()) == on_disk
