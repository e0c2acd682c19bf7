import os
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

import pe_pkg  # noqa: E402

pe_pkg.load()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the kernels through the C ABI")


@pytest.fixture(scope="session")
def pe():
    return sys.modules["photon_engine_b200"]


@pytest.fixture(scope="session")
def device(pe):
    dev = pe.create_device("cuda:0")
    if dev is None:
        pytest.fail("no CUDA device: GPU tests need a B200")
    yield dev
    dev.close()


@pytest.fixture(scope="session")
def oracle():
    import oracle as orc
    if not orc.available():
        pytest.skip("oracle/_ref/libphoton_ref.so not built (make -C oracle)")
    return orc
