import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


def _ensure_built():
    # build.py by path: the package import needs the library built here
    import importlib.util
    spec = importlib.util.spec_from_file_location("blest_b200_build", ROOT / "blest_b200" / "build.py")
    builder = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(builder)
    builder.build()
    import oracle
    if not oracle.ORACLE_SO.exists():
        oracle.build(ref=False)


_ensure_built()


def host_fixtures():
    return sorted(GOLDEN.glob("host_*.npz"))


@pytest.fixture(params=host_fixtures(), ids=lambda p: p.stem)
def host_golden(request):
    return dict(np.load(request.param, allow_pickle=False))


@pytest.fixture(scope="session")
def gpu():
    """Initialise the device once; GPU tests fail loudly without one."""
    import blest_b200
    blest_b200.init(0)
    return True
