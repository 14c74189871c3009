"""Shared fixtures. GPU tests are marked ``gpu`` and skipped without CUDA."""
import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden" / "reference_golden.npz"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def pytest_collection_modifyitems(config, items):
    try:
        import torch

        has_cuda = torch.cuda.is_available()
    except Exception:
        has_cuda = False
    if has_cuda:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def golden():
    return np.load(GOLDEN)


def golden_asset(z, name):
    """Reference robot asset (panda / fetch / baxter) from the golden file."""
    a = {k.split("/", 1)[1]: z[k] for k in z.files if k.startswith(name + "/")}
    out = {"name": name, "n_dof": int(a["n_dof"]), "n_joints": int(a["n_joints"])}
    for k in ("fixed_transforms", "joint_types", "spheres_flat", "sphere_to_joint", "self_cc_ranges_flat",
              "joint_lower", "joint_upper", "joint_parents", "joint_id_to_dof", "t_memory_idx", "dfs_order",
              "approx_spheres_flat", "approx_sphere_to_joint", "approx_self_cc_ranges_flat"):
        out[k] = a[k].tolist()
    return out, a
