import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_npz(name):
    z = np.load(GOLDEN / name)
    return {k: z[k] for k in z.files}


def unpack(z):
    off = z["offsets"]
    return [z["concat"][off[k]:off[k + 1]].tobytes() for k in range(len(off) - 1)]


@pytest.fixture(scope="session")
def kats():
    return json.loads((GOLDEN / "kat_pairs.json").read_text())


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.lib()
    return oracle
