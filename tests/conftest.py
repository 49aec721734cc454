import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests through the C ABI")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def golden_files():
    return np.load(os.path.join(GOLDEN, "reference_files.npz"))


@pytest.fixture(scope="session")
def golden_kat():
    return np.load(os.path.join(GOLDEN, "kat_maps.npz"))


@pytest.fixture(scope="session")
def golden_pairs():
    return np.load(os.path.join(GOLDEN, "pair_bundles.npz"))


@pytest.fixture(scope="session")
def golden_trunc():
    """tests/golden/truncated_lowest.npz: the reference's curvelet stage on the
    lowest-index neighbour lists of maps with truncated anchors."""
    return np.load(os.path.join(GOLDEN, "truncated_lowest.npz"))


def truncated_cases(z):
    """(case, scalar) pairs of truncated_lowest.npz."""
    return sorted({tuple(k.split("/")[:2]) for k in z.files if not k.startswith("pin_f32/")})


@pytest.fixture(scope="session")
def engine():
    import curvelet_construction_on_gpu_b200 as cvl
    eng = cvl.Engine()
    yield eng
    eng.close()
