"""Test configuration.

Marker ``gpu``: needs a CUDA device (a B200); everything else runs on CPU.
The CPU oracle (oracle/, test infrastructure) and the C-ABI library
(pyrowave_b200/libpyrowave-shared.so.0) are built on demand when a compiler is
available; on a machine that only received prebuilt files they are used as is.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    oracle_so = os.path.join(ROOT, "oracle", "liboracle.so")
    src = os.path.join(ROOT, "oracle", "pyrowave_oracle.cpp")
    if not os.path.exists(oracle_so) or os.path.getmtime(oracle_so) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=False)
    try:
        from pyrowave_b200 import build

        if subprocess.run(["which", "nvcc"], capture_output=True).returncode == 0 or os.path.exists("/usr/local/cuda/bin/nvcc"):
            build.build()
    except Exception as exc:  # the tests that need the library report the failure themselves
        sys.stderr.write(f"note: library build skipped: {exc}\n")


def cuda_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    if not cuda_available():
        pytest.skip("no CUDA device")
    import torch

    torch.cuda.init()
    return torch.device("cuda:0")
