import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")

def _reference_root() -> str:
    """The reference's source tree, as oracle/build_oracle.py locates it
    (CUPBR_REFERENCE_ROOT, else the recipe's default)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("_oracle_build_paths", os.path.join(ROOT, "oracle", "build_oracle.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.DEFAULT_REF


REFERENCE_ROOT = _reference_root()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN
