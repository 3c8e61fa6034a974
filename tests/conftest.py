import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: longer CPU case")


@pytest.fixture(scope="session")
def water():
    from stda_b200.molden import read_molden
    from stda_b200.integrals import ao_integrals
    mol = read_molden(os.path.join(GOLDEN, "water_sto3g.molden"))
    return mol, ao_integrals(mol)
