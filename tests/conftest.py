import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA library)")


@pytest.fixture(scope="session")
def oracle():
    from tests.oracle_bind import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def adb():
    import alliancedb_b200 as adb
    adb.lib()
    return adb
