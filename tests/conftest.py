"""Test configuration: the `gpu` marker selects tests that need a B200; everything else runs
on the CPU (oracle against golden vectors, host logic, C-ABI loading)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (run with -m gpu)")


def cuda_device_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
