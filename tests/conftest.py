"""Shared fixtures of the test suite.

Tests marked ``gpu`` need a CUDA device and the built library; the rest run
on any machine (no GPU) and cover the oracle, the configuration reader, the
file writers' host logic and the library's exported symbols.
"""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"
CONFIGS = GOLDEN / "configs"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU and the built CUDA library")


def has_gpu() -> bool:
    try:
        import mcml_gpu_b200 as m
        return m.device_count() > 0
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu_available():
    if not has_gpu():
        pytest.fail("this test needs a CUDA GPU and the built library")
    return True


def load_case(case: str):
    import mcml_gpu_b200 as m
    d = CONFIGS / case
    return m.parse_config(d / "sim_set.json", d / "input.txt")[0]
