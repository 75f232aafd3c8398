import glob
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")
REFERENCE_DIR = os.path.join(os.environ.get("CVRP_REFERENCE_DIR", "/root/reference"), "cvrp_ocl")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


def _ensure_built():
    # the oracle (checker) and the product library are built in-tree; on a GPU
    # box they arrive prebuilt with the repository snapshot
    orc = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(orc):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "liboracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    if os.path.isdir(REFERENCE_DIR) and not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libcvrp_ref.so")):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True, stdout=subprocess.DEVNULL)
    lib = os.path.join(ROOT, "cvrp_aco_ocl_b200", "libcvrp_aco.so")
    if not os.path.exists(lib):
        from cvrp_aco_ocl_b200 import build
        build.build()


_ensure_built()


def golden_cases():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    if not has_gpu():
        pytest.skip("no CUDA device")
    return 0
