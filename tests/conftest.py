"""Test configuration: the ``gpu`` marker, the package loader and the oracle.

Tests marked ``gpu`` need a B200 and call the product through its C ABI;
the rest run on the CPU (oracle pinning, ABI exports, host logic).
"""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def pkg():
    import __graft_entry__
    return __graft_entry__.load_package()


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle
    return oracle


@pytest.fixture(scope="session")
def ctx(pkg):
    c = pkg.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="session", params=["single_launch", "pass_loop"])
def ctx_any(pkg, request):
    """A context on each sort path: inputs that fit one wave of resident
    blocks in one cooperative launch, and the multi-launch pass loop."""
    c = pkg.Context(0)
    c.set_option(c.OPT_SINGLE_LAUNCH, 1 if request.param == "single_launch" else 0)
    yield c
    c.close()
