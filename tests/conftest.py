import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libqmbed_b200.so")


@pytest.fixture(scope="session")
def anchors():
    import json
    return json.loads((ROOT / "tests" / "golden" / "reference_anchors.json").read_text())


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as module
    module.build()
    return module
