import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

# the reference's real road graph: from the local, uncommitted copy under tests/golden/_data/ (the
# oracle Makefile's `fixtures` target writes it from a reference checkout), else from the checkout
# named by QBC_REFERENCE_DIR; the tests that need it skip when neither exists
_REF_DIR = os.environ.get("QBC_REFERENCE_DIR", "")


def _candidates(local, *rel):
    c = [os.path.join(GOLDEN, "_data", local)]
    if _REF_DIR:
        c.append(os.path.join(_REF_DIR, *rel))
    return c


LA_CANDIDATES = _candidates("LosAngeles.txt", "data", "roadData", "LosAngeles.txt")
LA_ORDER_CANDIDATES = _candidates("LosAngelesOrder.txt", "data", "orderFile", "LosAngelesOrder.txt")
LA_QUERY_CANDIDATES = _candidates("LosAngelesQuery.txt", "data", "queryBatch", "LosAngeles.txt")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _first(paths):
    for p in paths:
        if os.path.exists(p):
            return p
    return None


@pytest.fixture(scope="session")
def la_path():
    p = _first(LA_CANDIDATES)
    if p is None:
        pytest.skip("LosAngeles graph not available")
    return p


@pytest.fixture(scope="session")
def la_order_path():
    p = _first(LA_ORDER_CANDIDATES)
    if p is None:
        pytest.skip("LosAngeles order file not available")
    return p


@pytest.fixture(scope="session")
def la_query_path():
    p = _first(LA_QUERY_CANDIDATES)
    if p is None:
        pytest.skip("LosAngeles query batch not available")
    return p


@pytest.fixture(scope="session")
def g2k_path():
    return os.path.join(GOLDEN, "g2k.txt")


@pytest.fixture(scope="session")
def graph_cache(tmp_path_factory):
    return str(tmp_path_factory.mktemp("graphs"))


def rel_err(a, b):
    """Largest relative difference |a - b| / |b|.  Entries of b near zero are measured against a
    floor of 1e-12 * max|b| (a BC that is exactly 0 in b must be 0 in a up to that floor)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if not a.size:
        return 0.0
    floor = max(1e-12 * float(np.max(np.abs(b))), np.finfo(np.float64).tiny)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor)))
