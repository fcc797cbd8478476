import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle_pool():
    """Worker processes for oracle computations. Started with spawn, so that
    no worker is forked from a process that holds a CUDA context."""
    import multiprocessing as mp
    pool = mp.get_context("spawn").Pool(min(16, os.cpu_count() or 1))
    yield pool
    pool.close()
    pool.join()


@pytest.fixture(scope="session")
def ctx():
    from costuum_b200.tmatrix import Context
    c = Context(0)
    yield c
    c.close()
