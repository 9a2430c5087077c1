import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")

# the 20x20 seed-1 instance (Johnson bound, UB = optimum 2352): reference
# multicore counters measured with oracle/_ref/bbJ, 8 threads
CONFIG2 = dict(n=20, m=20, seed=1, opt=2352, decomposed=12616547, johnson_bounds=25431709,
               simple_bounds=236462768, leaves=0)


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
