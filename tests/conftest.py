import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
# compiled generated kernels are cached on disk; keep the tests' cache in the tree
os.environ.setdefault("SMG_JIT_CACHE_DIR", os.path.join(ROOT, "_build", "jit_cache"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running CPU test")
