import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("ghostz-gpu_b200", "oracle", "tests"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def params():
    from gzb import params as P
    return P.make_params()


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.build()
    return O.Oracle()


@pytest.fixture(scope="session")
def reference():
    import oracle as O
    if not os.path.exists(O.REF_LIB):
        O.build(ref=True)
    if not os.path.exists(O.REF_LIB):
        pytest.skip("reference units not built here (no reference checkout)")
    return O.Reference()
