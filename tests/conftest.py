"""Shared test setup: the `gpu` marker, import paths and in-tree builds.

CPU tests (-m "not gpu") cover the oracle against the golden fixtures, the host
generator, the C-ABI exports and the multi-rank host logic; GPU tests
(-m gpu) call the CUDA kernels through the C-ABI and compare with the oracle.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "hpccg-f90_b200")
for p in (ROOT, PKG, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def _ensure_built():
    if not os.path.exists(os.path.join(PKG, "libhpccg_b200.so")):
        subprocess.run(["make", "-s", "-j8", "-C", PKG], check=True)
    if not (os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so"))
            and os.path.exists(os.path.join(ROOT, "oracle", "liboracle_omp.so"))):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


_ensure_built()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if gpu_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)
