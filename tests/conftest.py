import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden" / "reference_cases.npz"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the sm_100a kernels)")


def golden_cases():
    data = np.load(GOLDEN)
    names = sorted({k.split("/")[0] for k in data.files})
    return {name: {f: data[f"{name}/{f}"] for f in
                   ("text", "sa", "isa", "lcp", "primary", "anchor_pos", "anchor_val")}
            for name in names}


@pytest.fixture(scope="session")
def golden():
    return golden_cases()


@pytest.fixture(scope="session")
def ctx():
    import sufkit_b200
    c = sufkit_b200.Context(0)
    yield c
    c.close()
