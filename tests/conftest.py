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


# Contract bars for floating-point results against the FP64 oracle.
COST_REL_TOL = 1e-5       # cost / clearance: |ours - fp64| / max(|fp64|, 1)
GRAD_REL_TOL = 1e-5       # gradient: relative L2 over the compared waypoints
MAX_KINK_EXCLUDED = 0.05  # at most this fraction of waypoints may be excluded


def kink_threshold(h):
    """A central difference with step h (rad) moves a sphere by at most about
    h times the longest lever arm (< 2 m on these robots); a waypoint closer
    than 10x that to a kink of the cost is not FD-comparable."""
    return 20.0 * h


def assert_gradient_vs_fd(ours, fd, kink, label, h=1e-6):
    """Relative L2 error of the adjoint gradient against FP64 central
    differences (step h) over the waypoints at least kink_threshold(h) from a
    kink of the state cost (hinge activation, min ties, box regions, ESDF
    voxel faces), with the excluded count bounded and each excluded
    waypoint's kink distance printed."""
    ok = kink > kink_threshold(h)
    excluded = np.nonzero(~ok)[0]
    num = np.linalg.norm((ours - fd)[ok])
    den = max(np.linalg.norm(fd[ok]), 1e-12)
    err = num / den
    print(f"{label}: rel L2 err vs FP64 FD (h={h:g}) = {err:.2e} over {ok.sum()} of {len(ok)} waypoints; "
          f"excluded {len(excluded)} (kink closer than {kink_threshold(h):g} m) with kink distances (m) "
          f"{np.array2string(np.sort(kink[excluded]), precision=1, max_line_width=400)}")
    assert len(excluded) <= MAX_KINK_EXCLUDED * len(ok), f"{len(excluded)} of {len(ok)} waypoints excluded"
    assert np.linalg.norm(fd[ok]) > 0
    assert err < GRAD_REL_TOL, f"{label}: {err:.2e}"
    return err
