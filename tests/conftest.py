"""Test configuration: the `gpu` marker and import paths.

Tests marked `gpu` need a B200 and call the CUDA library through its C ABI;
everything else runs on a CPU-only host."""
import os
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (REPO, os.path.join(REPO, "black-hole-simulator_b200"), os.path.join(REPO, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
