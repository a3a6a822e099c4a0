import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    # GPU tests are not skipped when no device is present: run `-m "not gpu"` on a
    # CPU-only machine, `-m gpu` on a B200.
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
