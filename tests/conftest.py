"""Shared test setup: markers, build of the oracle and of the CUDA library."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the oracle (and the reference library where its sources exist) and
    the product library if they are missing."""
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    # incremental: only sources newer than their objects are recompiled
    subprocess.run([sys.executable, "-m", "multi_species_b200.build"], cwd=ROOT, check=True,
                   stdout=subprocess.DEVNULL)
    yield


def gpu_available() -> bool:
    try:
        import multi_species_b200 as M
        f = M.E_MQ_DirectSum_B200(1.0, 0.1)
        f.close()
        return True
    except Exception:
        return False
