import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "tests" / "golden"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the engine library and the oracle once per session (no-ops when current)."""
    from cuda_multiddm_b200.build import build
    build()
    import subprocess
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "oracle"], check=True)
    yield


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available() and torch.cuda.get_device_capability(0)[0] == 10
    except Exception:
        return False
