"""Shared pytest setup: import paths and the ``gpu`` marker.

Tests marked ``gpu`` need a CUDA device and the built library; everything else
runs on a CPU-only machine.
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "momentumed.jl_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libmomed_b200.so")
