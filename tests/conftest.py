import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "endless-games-of-war_b200")
ORACLE = os.path.join(ROOT, "oracle")
for p in (PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        g = json.load(f)

    def intkeys(d):
        if isinstance(d, dict):
            out = {}
            for k, v in d.items():
                try:
                    k = int(k)
                except (TypeError, ValueError):
                    pass
                out[k] = intkeys(v)
            return out
        if isinstance(d, list):
            return [intkeys(x) for x in d]
        return d
    return intkeys(g)


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def wl():
    """warlib with a CUDA device; GPU tests only."""
    import warlib
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test without a CUDA device")
    warlib.lib()
    return warlib
