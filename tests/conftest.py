import json
import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (sm_100a) and libbugdef.so")


def pytest_collection_modifyitems(config, items):
    # run the no-allocation entry-point test file last when present
    items.sort(key=lambda it: 1 if "test_zz_" in str(it.fspath) else 0)


@pytest.fixture(scope="session")
def golden():
    def load(name):
        if name.endswith(".json"):
            with open(GOLDEN / name) as f:
                return json.load(f)
        return np.load(GOLDEN / name, allow_pickle=False)
    return load


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import bug_defense_b200 as bd
    from bug_defense_b200 import build
    build.build()
    return bd
