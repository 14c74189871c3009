"""The C ABI from a C++ caller (tests/cabi_demo/edge_bridge_demo.cpp), the way
the reference's C++ planners hold EdgeEvalGpu (edge_batch_bridge.hh:27-111):
model from descriptor arrays, a scene of device OBB arrays, the host-buffer
edge bridge. CPU: the program compiles and links against include/prism_b200.h
and the library. GPU: its verdicts and costs equal the Python path's and the
reference kernels' bit for bit."""
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from prismplan_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "cabi_demo" / "edge_bridge_demo.cpp"
CUDA = Path("/usr/local/cuda")


def _build(out_dir: Path) -> Path:
    cxx = shutil.which("g++")
    if cxx is None or not (CUDA / "include" / "cuda_runtime.h").is_file():
        pytest.skip("no g++ or CUDA headers")
    exe = out_dir / "edge_bridge_demo"
    cmd = [cxx, "-std=c++17", "-O2", "-Wall", "-Werror", f"-I{ROOT / 'include'}", f"-I{CUDA / 'include'}", str(SRC),
           f"-L{_lib.LIB_PATH.parent}", "-lprism_b200", f"-L{CUDA / 'lib64'}", "-lcudart",
           f"-Wl,-rpath,{_lib.LIB_PATH.parent}", "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_cpp_caller_compiles_and_links(tmp_path):
    exe = _build(tmp_path)
    assert exe.is_file()


def _write_problem(path: Path, b, obbs, frm, to, step, max_samples):
    def i32(*v):
        return np.asarray(v, np.int32).tobytes()

    def arr(values, dt):
        return np.ascontiguousarray(np.asarray(values, dt)).tobytes()

    tree = len(b.joint_parents) == b.n_joints and b.n_joints > 0
    dims, pose, en = obbs
    n_o = len(en)
    en_p = np.zeros((n_o + 3) // 4 * 4, np.uint8)
    en_p[:n_o] = en
    parts = [i32(0x50534231, b.n_dof, b.n_joints, len(b.sphere_to_joint), len(b.self_cc_ranges_flat) // 3,
                 len(b.approx_sphere_to_joint), len(b.approx_self_cc_ranges_flat) // 3, int(tree), n_o, len(frm),
                 max_samples),
             np.float32(step).tobytes(),
             arr(b.fixed_transforms, np.float32), arr(b.joint_types, np.int32), arr(b.spheres_flat, np.float32),
             arr(b.sphere_to_joint, np.int32), arr(b.self_cc_ranges_flat, np.int32),
             arr(b.approx_spheres_flat, np.float32), arr(b.approx_sphere_to_joint, np.int32),
             arr(b.approx_self_cc_ranges_flat, np.int32), arr(b.joint_lower, np.float32),
             arr(b.joint_upper, np.float32)]
    if tree:
        parts += [arr(b.joint_parents, np.int32), arr(b.joint_id_to_dof, np.int32), arr(b.t_memory_idx, np.int32),
                  arr(b.dfs_order, np.int32)]
    parts += [arr(dims, np.float32), arr(pose, np.float32), en_p.tobytes(), arr(frm, np.float32), arr(to, np.float32)]
    path.write_bytes(b"".join(parts))


@pytest.mark.gpu
def test_cpp_caller_matches_python_and_reference(tmp_path):
    import torch

    import oracle
    from prismplan_b200 import api, workloads
    from prismplan_b200.robot import RobotModelBuilder
    from prismplan_b200.scene import SceneTensors

    exe = _build(tmp_path)
    wl = workloads.workload(2, scale=1.0 / 16)   # 4096 edges, Panda-like chain, 64 OBBs
    b = RobotModelBuilder.from_asset(wl["asset"])
    frm, to = wl["from"], wl["to"]
    prob, out = tmp_path / "problem.bin", tmp_path / "out.bin"
    _write_problem(prob, b, wl["obbs"], frm, to, 0.01, 600)
    res = subprocess.run([str(exe), str(prob), str(out)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    raw = out.read_bytes()
    E = len(frm)
    valid = np.frombuffer(raw[:E], np.uint8)
    cost = np.frombuffer(raw[E:], np.float32)
    b.build()
    sc = SceneTensors(*wl["obbs"])
    p = api.EdgeEvalParams(max_joint_step=0.01, max_samples=600)
    v, c, _ = api.check_edges(b, sc, torch.from_numpy(frm).cuda(), torch.from_numpy(to).cuda(), params=p)
    np.testing.assert_array_equal(valid, v.cpu().numpy())
    assert np.array_equal(cost.view(np.uint32), c.cpu().numpy().view(np.uint32))
    ref = oracle.RefKernels(b, *wl["obbs"])
    rv, rc, _ = ref.check_edges(frm, to, wl["G"])
    np.testing.assert_array_equal(valid, rv)
    assert np.array_equal(cost.view(np.uint32), rc.view(np.uint32))
    assert 0.0 < valid.mean() < 1.0
    print(res.stdout.strip())
