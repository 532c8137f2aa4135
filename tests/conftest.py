import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def si8():
    from qxmd_b200 import cell
    return cell.si8()


@pytest.fixture(scope="session")
def si8_psi(si8):
    """Orthonormalised initial wavefunctions of Si8 (reference LCG, seed 25)."""
    import oracle
    from qxmd_b200 import cell
    c = cell.random_wavefunctions(si8.gs.nplwex, si8.nband)
    c, _, rc = oracle.schmidt(c)
    assert rc == 0
    return c
