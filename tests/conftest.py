import os
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA path through the C-ABI")


def _ensure_built():
    """The product library and the oracle are built in-tree; build them if this checkout has not yet."""
    from raytracing_b200 import build as product_build
    from oracle import binding

    if not product_build.LIBRARY.exists() and os.environ.get("RT_B200_NO_BUILD") is None:
        product_build.build()
    if not binding.LIBRARY.exists():
        binding.build()


_ensure_built()


@pytest.fixture(scope="session")
def rt():
    import raytracing_b200

    return raytracing_b200


@pytest.fixture(scope="session")
def oracle():
    from oracle import binding

    binding.load()
    return binding
