import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA library")
    config.addinivalue_line("markers", "slow: long-running")


def _ensure_built():
    import _oracle

    if not os.path.exists(_oracle.LIB):
        _oracle.build()
    from proresraw_rs_b200 import build

    need = [os.path.join(ROOT, "proresraw_rs_b200", "lib", n) for n in ("libprr.so", "libprr_synth.so")]
    if not all(os.path.exists(p) for p in need):
        build.build()


_ensure_built()
