import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) CUDA device")
    config.addinivalue_line("markers", "slow: long-running parity case")
    # temporary files of the tests stay inside the repository (git-ignored)
    if not config.option.basetemp:
        config.option.basetemp = os.path.join(ROOT, "tests", "_tmp")


@pytest.fixture(scope="session")
def oracles():
    """(reference C oracle or None, C restatement) -- built on demand."""
    from oracle import build as obuild
    from oracle import lib as olib
    obuild.build_cmsm()
    ref = None
    try:
        obuild.build_all()
    except Exception:
        pass
    if os.path.exists(olib.REF_LIB):
        ref = olib.RefOracle()
    return ref, olib.COracle()


@pytest.fixture(scope="session")
def zlib():
    from zkmetal_b200 import build as zbuild
    if not zbuild.up_to_date():
        zbuild.build()
    from zkmetal_b200 import lib as zl
    return zl.lib()
