import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)
GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


def golden_cases(prefix="engine_"):
    return sorted(f[len(prefix):-4] for f in os.listdir(GOLDEN) if f.startswith(prefix) and f.endswith(".npz"))


@pytest.fixture(scope="session")
def golden():
    from lightsmith_b200 import plan as P

    cache = {}

    def load(name):
        if name not in cache:
            cache[name] = P.load(os.path.join(GOLDEN, name + ".npz"))
        return cache[name]
    return load
