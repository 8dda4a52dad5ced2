"""pytest configuration: the `gpu` marker and import paths.

`-m gpu` tests call the CUDA kernels through the C-ABI (libgdiamond_b200.so) and need a GPU;
everything else runs on the CPU.  The CPU oracle (oracle/) is the checker in both.
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
