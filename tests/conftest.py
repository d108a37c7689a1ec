import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TESTS = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(TESTS, "golden")
for p in (ROOT, TESTS):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA path through the C ABI")
    config.addinivalue_line("markers", "slow: longer statistical checks")


@pytest.fixture(scope="session")
def oracle():
    from ltref import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def golden4():
    return dict(np.load(os.path.join(GOLDEN, "ref_4x4x4x4.npz")))


@pytest.fixture(scope="session")
def golden_odd():
    return dict(np.load(os.path.join(GOLDEN, "ref_4x6x8x10.npz")))


@pytest.fixture(scope="session")
def golden_bias():
    return dict(np.load(os.path.join(GOLDEN, "ref_bias.npz")))


@pytest.fixture(scope="session")
def golden_bmw():
    d = dict(np.load(os.path.join(GOLDEN, "ref_bmw.npz")))
    d["two_row_file"] = os.path.join(GOLDEN, "ref_2x4x6x8.bmw")
    return d


@pytest.fixture(scope="session")
def golden_measure(oracle):
    """Reference measurement bundle and flow samples; "U" is the regenerated input."""
    from ltref import haar_links_numpy
    d = dict(np.load(os.path.join(GOLDEN, "ref_measure.npz")))
    ext = tuple(int(e) for e in d["ext"])
    d["U"] = oracle.heatbath(ext, haar_links_numpy(ext, 2), 6.0, 5, 17, 0)
    return d


@pytest.fixture(scope="session")
def golden_md(oracle):
    """Reference MD integrators and parity update; "U" and "P" are the regenerated inputs."""
    from ltref import haar_links_numpy
    d = dict(np.load(os.path.join(GOLDEN, "ref_md.npz")))
    ext = tuple(int(e) for e in d["ext"])
    d["U"] = oracle.heatbath(ext, haar_links_numpy(ext, 2), 6.0, 5, 17, 0)
    d["P"] = oracle.random_momenta(ext, 9, 0)
    return d


@pytest.fixture(scope="session")
def golden_rect(oracle):
    """Reference Rectangular<2> staples, Checkerboard4 overrelaxation, MD and flow on 8^4; "U"
    and "P" are the regenerated inputs."""
    from ltref import haar_links_numpy
    d = dict(np.load(os.path.join(GOLDEN, "ref_rect.npz")))
    ext = tuple(int(e) for e in d["ext"])
    d["U"] = oracle.heatbath(ext, haar_links_numpy(ext, 4), 6.0, 3, 21, 0)
    d["P"] = oracle.random_momenta(ext, 9, 0)
    return d


@pytest.fixture(scope="session")
def golden_chain():
    return dict(np.load(os.path.join(GOLDEN, "ref_chain_8x8x8x8.npz")))
