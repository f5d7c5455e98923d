"""Shared test setup.

GPU tests carry @pytest.mark.gpu and run on a B200; everything else runs on the CPU. The
reference library (oracle/_ref) and the oracle restatement (oracle/_build) are the checkers; the
product is hnsw_vector_search_b200/libvdx_b200.so, built in-tree.
"""

import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    import hnsw_vector_search_b200.build as b
    b.build()
    import oracle as o
    if not o.ORACLE_LIB.exists():
        o.build(ref=False)
    yield


@pytest.fixture(scope="session")
def vdx():
    import hnsw_vector_search_b200 as v
    return v


@pytest.fixture(scope="session")
def orc():
    import oracle as o
    return o


def has_gpu() -> bool:
    try:
        import hnsw_vector_search_b200 as v
        return v.device_count() > 0
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu(vdx):
    if vdx.device_count() == 0:
        pytest.fail("no CUDA device: GPU tests must run on a GPU")
    return vdx


def integer_matrix(rows, dim, seed):
    """The reference's portable fixture (tests/hnsw_parallel_test.cpp:37-48)."""
    import oracle as o
    return o.Oracle().integer_matrix(rows, dim, seed)


def uniform_matrix(rows, dim, seed, lo=-1.0, hi=1.0):
    return np.random.default_rng(seed).uniform(lo, hi, size=(rows, dim)).astype(np.float32)
