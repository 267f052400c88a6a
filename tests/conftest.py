import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("", "oracle", "icp-gpu_b200", "icp-gpu_b200/csrc", "tests"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _ensure_built():
    """Build the oracle and the library in-tree if they are missing (no-op when
    the prebuilt .so files travelled with the repository)."""
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle_cpu.so")):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    if not os.path.exists(os.path.join(ROOT, "icp-gpu_b200", "libbls_gpu.so")):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "icp-gpu_b200")])


_ensure_built()


@pytest.fixture(scope="session")
def golden():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "reference_vectors.json")) as f:
        g = json.load(f)
    import numpy as np
    return {k: np.array([int(h, 16) for h in v["limbs"]], dtype=np.uint64)
            for k, v in g.items() if isinstance(v, dict) and "limbs" in v}
