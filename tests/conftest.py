import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (B200)")


def load_golden(kind: str):
    z = np.load(os.path.join(GOLDEN, f"tiny_{kind}.npz"))
    return {k: z[k] for k in z.files}


def golden_tree(g):
    from oracle.pyoracle import Tree
    return Tree(g["bounds"], g["child"], g["children"], g["axis"], g["left_cheaper"], g["ids"])


def golden_mesh(g):
    from rfmanta_b200.scenes import Mesh
    return Mesh(g["vertices"], g["indices"], g["face_material"], g["materials"])


@pytest.fixture(scope="session")
def restatement():
    from oracle.pyoracle import Restatement
    return Restatement()


@pytest.fixture(scope="session", params=["wald", "ks"])
def golden(request):
    return request.param, load_golden(request.param)


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
