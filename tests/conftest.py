import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    # Build the product library and the CPU checker if they are missing (the
    # snapshot normally carries prebuilt copies).
    for mk, out in (("rayengine_b200/csrc/Makefile", "rayengine_b200/librayengine_b200.so"),
                    ("oracle/Makefile", "oracle/liboracle.so")):
        if not os.path.exists(os.path.join(ROOT, out)):
            subprocess.run(["make", "-j8", "-f", os.path.join(ROOT, mk)], cwd=ROOT, check=True)


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    return torch.device("cuda:0")
