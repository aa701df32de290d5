"""Test setup: import paths for the library package (g2-aimd_b200/g2aimd) and
the CPU oracle (oracle/), the `gpu` marker, and shared graph fixtures."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "g2-aimd_b200"), os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libg2aimd.so")


@pytest.fixture(scope="session")
def g2():
    import g2aimd
    g2aimd.lib()
    return g2aimd


@pytest.fixture(scope="session")
def orc():
    import orc as _orc
    _orc.lib()
    return _orc


@pytest.fixture(scope="session")
def c1_graph(g2):
    """ER(2000, 0.01) + 5 planted K12, ids in degeneracy order."""
    return g2.Graph.er(2000, 0.01, planted=5, planted_size=12, seed=7).degeneracy_recoded()


@pytest.fixture(scope="session")
def ctx(g2):
    from g2aimd.context import Context
    c = Context(0)
    yield c
    c.close()
