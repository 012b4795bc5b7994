import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O
    O.lib()
    return O


_TABLE_CACHE = {}


@pytest.fixture(scope="session")
def table_cache(oracle_mod):
    """Leaf tables keyed by the parameters they depend on."""
    def get(**kw):
        p = oracle_mod.params(**kw)
        key = (p.n_cheb, p.kappa, p.degree, p.L, p.depth)
        if key not in _TABLE_CACHE:
            _TABLE_CACHE[key] = oracle_mod.tables(p)
        return p, _TABLE_CACHE[key]
    return get
