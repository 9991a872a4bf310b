import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

import __graft_entry__ as ge  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests proper")
    config.addinivalue_line("markers", "slow: larger parity cases")


@pytest.fixture(scope="session")
def pkg():
    return ge.load_package()


@pytest.fixture(scope="session")
def orc():
    return ge.load_oracle()


@pytest.fixture(scope="session")
def oracle(orc):
    return orc.Oracle()


@pytest.fixture(scope="session")
def ref_host(orc):
    if not orc.available("ref_host"):
        pytest.skip("reference host build absent")
    return orc.RefHost()


@pytest.fixture(scope="session")
def cuda_ok():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ctx(pkg, cuda_ok):
    if not cuda_ok:
        pytest.skip("no CUDA device")
    return pkg.Context(0)


@pytest.fixture(scope="session")
def ref_gpu(orc, cuda_ok):
    if not cuda_ok:
        pytest.skip("no CUDA device")
    if not orc.available("ref_gpu"):
        pytest.fail("oracle/_ref/libppfref_gpu.so missing: build it with `make -C oracle ref`")
    return orc.RefGPU()
