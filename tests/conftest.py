import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU")


def _has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def built_library():
    from cctag_b200.build import build_library

    return build_library()


@pytest.fixture(scope="session")
def orc():
    import oracle

    oracle.build_oracle()
    oracle.load()
    return oracle


@pytest.fixture(scope="session")
def golden_tables():
    return dict(np.load(GOLDEN / "reference_tables.npz"))


@pytest.fixture(scope="session")
def opencv_cases():
    return dict(np.load(GOLDEN / "opencv_cases.npz"))


@pytest.fixture(scope="module")
def detector(built_library):
    import cctag_b200

    d = cctag_b200.Detector(max_w=3840, max_h=2160)
    yield d
    d.close()
