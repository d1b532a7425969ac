import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
ASSETS = os.path.join(ROOT, "assets")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def golden_asset(name):
    return os.path.join(GOLDEN, "assets", name + ".vbtp")


def generated_asset(name):
    """Path of a generated asset under assets/ (made by tests/golden/make_assets.py); skip if absent."""
    p = os.path.join(ASSETS, name + ".vbtp")
    if not os.path.exists(p):
        pytest.skip(f"asset {name} not generated (python tests/golden/make_assets.py {name})")
    return p


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle.oracle import REF_SO, Reference
    if not os.path.exists(REF_SO):
        pytest.skip("reference build (oracle/_ref) not present")
    return Reference()


@pytest.fixture(scope="session")
def vbt():
    import vbt_b200
    return vbt_b200


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch
