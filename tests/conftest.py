import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the sm_100a kernels)")
    # the checker (oracle restatement) is plain C: build it if missing
    if not os.path.exists(os.path.join(ROOT, "oracle", "liborc.so")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    # the product library: build it if missing (nvcc cross-compiles without a GPU)
    if not os.path.exists(os.path.join(ROOT, "dvbrx_b200", "libdvbrx_b200.so")):
        from dvbrx_b200 import build
        build.build()


@pytest.fixture(scope="session")
def golden():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "cases.json")) as f:
        return json.load(f)["cases"]
