import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "shape-cuda-v1.2_b200", "python"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _ensure_built():
    import subprocess
    if not os.path.exists(os.path.join(REPO, "oracle", "liboracle.so")):
        subprocess.run(["bash", os.path.join(REPO, "oracle", "build_oracle.sh")], check=True)
    lib = os.path.join(REPO, "shape-cuda-v1.2_b200", "lib", "libshape_b200.so")
    if not os.path.exists(lib):
        subprocess.run([sys.executable, os.path.join(REPO, "shape-cuda-v1.2_b200", "build.py")], check=True)


_ensure_built()


@pytest.fixture(scope="session")
def oracle():
    from oracle.bindings import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return 0
