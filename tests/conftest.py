import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "oracle", "ref"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built CUDA library")
    config.addinivalue_line("markers", "slow: long-running")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def sed_lib():
    """The CUDA library; GPU tests fail (not skip) if it is missing on a machine with a GPU."""
    if not gpu_available():
        pytest.skip("no CUDA device")
    from pubsed_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        _lib.build()
    return _lib.lib()


@pytest.fixture(scope="session")
def oracle():
    import oracle_lib
    return oracle_lib.oracle_lib()


def pytest_sessionfinish(session, exitstatus):
    """With SED_STATE_LOG set, the per-call outcomes of
    oracle_lib.check_states (packets compared, packets over 1e-12, largest
    difference) are written there as JSON."""
    path = os.environ.get("SED_STATE_LOG")
    if not path:
        return
    import json
    import oracle_lib
    with open(path, "w") as f:
        json.dump([{"test": t, "n": n, "n_over": k, "max": m} for t, n, k, m in oracle_lib.STATE_LOG], f, indent=0)
