import os
import sys


ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, 'tests', 'golden')
if GOLDEN not in sys.path:
    sys.path.insert(0, GOLDEN)


def _build_library_if_missing():
    """A fresh checkout has no liblc3d.so: build it (nvcc, sm_100a) before
    any test imports the package, which needs the library. The build module
    is loaded on its own, since importing the package loads the library."""
    import importlib.util
    path = os.path.join(ROOT, 'lcode3d_b200', 'build.py')
    spec = importlib.util.spec_from_file_location('lc3d_build_for_tests', path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    if not os.path.exists(mod.LIB):
        mod.build()


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA GPU (B200, sm_100a)')
    _build_library_if_missing()
