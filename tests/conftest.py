import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")

def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_golden(name):
    path = os.path.join(GOLDEN, name)
    if not os.path.exists(path):
        pytest.skip("golden fixture %s missing" % name)
    with open(path) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def bounds_golden():
    return load_golden("bounds_golden.json")


@pytest.fixture(scope="session")
def search_golden():
    return load_golden("search_golden.json")


@pytest.fixture(scope="session")
def sorted_golden():
    return load_golden("sorted_golden.json")


@pytest.fixture(scope="session")
def config2_golden(search_golden):
    """The second configuration (20x20 seed 1, weak then Johnson, UB = optimum
    2352): the reference multicore's counters, written into
    search_golden.json by `make_golden.py --big-only`."""
    big = [r for r in search_golden["runs"] if r.get("big")]
    if not big:
        pytest.skip("search_golden.json has no config-2 entry (make_golden.py --big-only)")
    return big[0]
