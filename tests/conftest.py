"""Test configuration: the `gpu` marker and import paths.

Tests marked gpu run the CUDA path on a B200; everything else runs on CPU
(the oracle against the reference's golden vectors, host logic, the C ABI's
exported symbols).
"""

import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
PACKAGE_ROOT = REPO / "pursuit-evasion-core_b200"
for path in (str(PACKAGE_ROOT), str(REPO)):
    if path not in sys.path:
        sys.path.insert(0, path)


def pytest_configure(config):
    config.addinivalue_line(
        "markers", "gpu: needs a CUDA GPU (B200) and the built libpe_b200.so"
    )


@pytest.fixture(scope="session")
def oracle():
    from tests import oracle_lib

    return oracle_lib.load()
