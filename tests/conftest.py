"""Test configuration: registers the `gpu` marker and puts the repo on sys.path.

`-m "not gpu"` runs the oracle pins, the known-answer tests, the host logic and
the C-ABI export checks on CPU; `-m gpu` runs the parity tests of the CUDA path
against the oracle on a B200.
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the CUDA path)")
    config.addinivalue_line("markers", "slow: oracle runs of tens of seconds")
