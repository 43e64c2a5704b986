"""pytest configuration: the `gpu` marker and import paths.

    python -m pytest tests -m "not gpu"   # oracle, host logic, ABI (CPU)
    python -m pytest tests -m gpu         # CUDA parity against the oracle
"""
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
for p in (HERE.parent, HERE, HERE / "golden"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the sm_100a kernels)")
