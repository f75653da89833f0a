import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

import __graft_entry__ as ge  # noqa: E402

ge.load_package()

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a library)")


@pytest.fixture(scope="session")
def ar():
    return ge.load_package()


@pytest.fixture(scope="session")
def O():
    from oracle import oracle

    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def gpu_lib(ar):
    ge._load_build_ext().build()
    return ar._lib.default_context()


class Golden:
    """Accessor for a packed golden .npz: g[case][array], g.meta[case]."""

    def __init__(self, path: Path):
        self.z = np.load(path)
        self.meta = json.loads(bytes(self.z["__meta__"]).decode())

    def cases(self, prefix=""):
        return sorted({k.split("::")[0] for k in self.z.files if "::" in k and k.startswith(prefix)})

    def __getitem__(self, case):
        return {k.split("::")[1]: self.z[k] for k in self.z.files if k.startswith(case + "::")}


@pytest.fixture(scope="session")
def ref_golden():
    return Golden(GOLDEN / "reference_fixtures.npz")


@pytest.fixture(scope="session")
def cv_golden():
    return Golden(GOLDEN / "opencv_golden.npz")


def fields(pts):
    """A PointSet as the mapping the oracle's track() takes."""
    from autorift_b200.points import FIELDS

    return {n: getattr(pts, n) for n in FIELDS}
