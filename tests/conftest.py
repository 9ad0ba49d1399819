"""Test setup: the package and the oracle on sys.path, the `gpu` marker, and shared fixtures."""

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
for p in (ROOT / "option-pricing-lab_b200", ROOT / "oracle", ROOT):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built engine library")
    config.addinivalue_line("markers", "slow: longer CPU checks")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle import Reference, reference_available

    if not reference_available():
        pytest.skip("the reference's CPU engine is not built here (make -C oracle ref needs the reference tree)")
    return Reference()
