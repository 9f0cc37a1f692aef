import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a kernels")


@pytest.fixture(scope="session")
def port():
    import oracle
    return oracle.Port()


@pytest.fixture(scope="session")
def ref():
    import oracle
    if not oracle.reference_available():
        pytest.skip("oracle/_ref/libcudaee_ref.so not built (needs the reference sources)")
    return oracle.Reference()


@pytest.fixture(scope="session")
def ctx():
    from cudaedgeelimination_b200 import Context, device_count
    assert device_count() > 0, "GPU tests need a CUDA device"
    c = Context(0)
    yield c
    c.close()
