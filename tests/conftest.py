import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the libdroplet.so kernels")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the oracle (gcc) and the CUDA library (nvcc cross-compiles without a GPU)."""
    import oracle as orc
    orc.build()
    from mpi_2d_domain_decomp_turb_particles_b200 import build_ext
    build_ext.build()
    yield
