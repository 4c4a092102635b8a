import os
import sys
import tempfile

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# The autotuner's user cache: a per-session file, so that tests neither read
# nor change the caches of whoever runs them. The shipped table (measured
# entries that change as the kernels are retuned) is left out, so that tests
# of the library's own shape rules see those rules; tests/test_tune_table.py
# checks the shipped table itself.
os.environ.setdefault("PHYSIS_B200_TUNE_CACHE",
                      os.path.join(tempfile.mkdtemp(prefix="physis_b200_tune_"), "tune.json"))
os.environ.setdefault("PHYSIS_B200_TUNE_SHIPPED", "0")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs on the GPU box)")
