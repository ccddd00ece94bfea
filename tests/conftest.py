"""Test configuration: the `gpu` marker and import paths.

Tests marked `gpu` need a B200 and call the CUDA library through its C ABI;
everything else runs on the CPU (the oracle, the host code, the ABI's exports,
the multi-rank plumbing over gloo).
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); calls the sm_100a library")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA GPU in this container")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def ccmod():
    import cosmic_collisions_b200 as cc
    from importlib import import_module
    import_module("cosmic_collisions_b200.build").build()
    return cc
