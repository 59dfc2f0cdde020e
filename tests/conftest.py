import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


def _ensure_built():
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libquest_ref.so")):
        # the reference's own sources, where a checkout exists (skipped otherwise)
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=False)
    if not (os.path.exists(os.path.join(ROOT, "quest_b200", "libquest_gpu.so")) and
            os.path.exists(os.path.join(ROOT, "quest_b200", "quest-gpu"))):
        subprocess.run(["make", "-s", "-j4", "-C", os.path.join(ROOT, "quest_b200", "csrc")], check=True)


_ensure_built()


@pytest.fixture(scope="session")
def golden_weights():
    from quest_b200.inputs import load_pc_weights
    return load_pc_weights(os.path.join(GOLDEN, "pc_weights_18_22_3.15.txt"))


@pytest.fixture(scope="session")
def oracle_weights(golden_weights):
    from oracle import oracle as O
    return O.Weights(*golden_weights)


def rel_err(ref: np.ndarray, got: np.ndarray) -> float:
    """max |got - ref| / max |ref| (the parity metric for one of rho00 / rho01)."""
    scale = float(np.abs(ref).max())
    diff = float(np.abs(got - ref).max())
    if scale == 0.0:
        return diff
    return diff / scale
