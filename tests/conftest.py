import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA engine")


def load_golden(name: str) -> dict:
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    out = {k: z[k] for k in z.files}
    if "meta" in out:
        out["meta"] = json.loads(str(out["meta"]))
    return out


WALK_CASES_CHAIN = ["walk_L16D16_DW16", "walk_L10D8_DW4", "walk_L10D8_DW2_branch", "walk_L10D8_DW1_branch",
                    "walk_debug_DW2", "walk_L10D8_DW4_field"]
WALK_CASES_2D = ["walk_snake3x3_D8_DW4", "walk_snake3x3_D8_DW4_field", "walk_snake4x4_D16_DW8_branch"]
WALK_CASES = WALK_CASES_CHAIN + WALK_CASES_2D


def couplings(z: dict):
    """(ci, cj, cJ) of a walk fixture: the reference's own coupling list when it was saved, else the
    open chain."""
    if "coup_i" in z:
        return z["coup_i"].astype(np.int32), z["coup_j"].astype(np.int32), z["coup_J"].astype(np.float64)
    L = z["meta"]["L"]
    ci = np.arange(L - 1, dtype=np.int32)
    return ci, ci + 1, np.ones(L - 1)


@pytest.fixture(scope="session")
def golden():
    return load_golden
