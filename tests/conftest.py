"""Test configuration.

GPU tests are marked ``gpu``; everything else runs on the CPU.  The oracle
libraries (oracle/liboracle.so and, where the reference sources are present,
oracle/_ref/) are built on first use if missing.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU")
    config.addinivalue_line("markers", "slow: longer CPU oracle runs")


def _ensure_oracle():
    port = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(port):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "port"], check=True,
                       stdout=subprocess.DEVNULL)


_ensure_oracle()


def ref_available(kind="bm1d") -> bool:
    return os.path.exists(os.path.join(ROOT, "oracle", "_ref", f"libref_{kind}.so"))


@pytest.fixture(scope="session")
def gpu_available():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True
