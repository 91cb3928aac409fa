import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def built():
    """libamj.so and the oracle libraries, built in-tree if absent."""
    import subprocess
    lib = os.path.join(ROOT, "accmultiwayjoins_b200", "libamj.so")
    orc = os.path.join(ROOT, "oracle", "liborc.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-C", os.path.join(ROOT, "accmultiwayjoins_b200", "csrc"), "-j8"], check=True)
    if not os.path.exists(orc):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True)
    return True


@pytest.fixture(scope="session")
def ctx(built):
    from accmultiwayjoins_b200 import Context
    c = Context(0)
    yield c
    c.close()
