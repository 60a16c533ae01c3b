"""Shared test configuration.

Markers: ``gpu`` -- needs a CUDA device (the parity tests proper, run on a
B200 with ``-m gpu``); everything else runs on the CPU.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    """The reference library when built (oracle/_ref), else the C restatement."""
    from oracle.oracle import best_available
    return best_available()


@pytest.fixture(scope="session")
def port_oracle():
    from oracle.oracle import Oracle
    return Oracle("port")


@pytest.fixture(scope="session")
def ref_oracle():
    from oracle.oracle import Oracle, available
    if not available("ref"):
        pytest.skip("reference library not built (make -C oracle ref needs the reference sources)")
    return Oracle("ref")
