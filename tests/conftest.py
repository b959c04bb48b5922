import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running oracle check")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def lib():
    """The C-ABI library, loaded through the package's ctypes binding."""
    from spectral_solver_b200 import _lib
    return _lib.load()


def golden_finals() -> dict:
    """The reference's published FP64 t = 20 finals (tests/golden/benchmark_finals.json,
    extracted from its Benchmark.md by tests/golden/make_golden.py), keyed by N."""
    import json
    with open(os.path.join(ROOT, "tests", "golden", "benchmark_finals.json")) as f:
        return {r["n"]: r for r in json.load(f)["runs"]}
