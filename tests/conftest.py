import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (sm_100a) and the built library")
    config.addinivalue_line("markers", "slow: long-running case")


def golden_cases():
    # step cases only; e9_* hold the isotropy protocol's restart series
    return sorted(p.stem for p in GOLDEN.glob("*.npz") if not p.stem.startswith("e9_"))


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN
