import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (HERE, ROOT, os.path.join(ROOT, "hyqmom.jl_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: longer CPU cases")


import pytest  # noqa: E402


@pytest.fixture(autouse=True)
def _device_errors_stay_with_their_test(request):
    """After a GPU test, wait for the device: an asynchronous device error then
    fails the test whose kernels raised it, not the next one."""
    yield
    if request.node.get_closest_marker("gpu") is None or "torch" not in sys.modules:
        return
    torch = sys.modules["torch"]
    if torch.cuda.is_available() and torch.cuda.is_initialized():
        torch.cuda.synchronize()
