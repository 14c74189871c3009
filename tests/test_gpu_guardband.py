"""GPU: the fast sphere-vs-box path and its guard band, pinned directly.

Every Boolean decides a pair with a 3x3 fast map first and falls back to the
reference's exact quaternion sequence (transform_sphere_to_local +
sphere_single_obb_collision, scene_collision.cuh:24-78) only when the fast
squared distance lands inside a guard band of (S + B + 1) * 2^-15 metres.
These tests hold that split to the reference's own kernels, bitwise, far from
the scales of the workloads: boxes 5-20 m from the origin, full extents up to
4 m (pairs) and 2 m (scenes), and stored quaternions up to 1e-3 off unit norm (the library builds its
fast matrix from the stored quaternion as it is, which is the map the
reference applies).
"""
import numpy as np
import pytest
import torch

import oracle
from prismplan_b200 import _lib, api, workloads
from prismplan_b200.robot import RobotModelBuilder
from prismplan_b200.scene import SceneTensors

pytestmark = pytest.mark.gpu


def _shell_boxes(rng, n, centre, r_lo, r_hi, half_lo, half_hi, quat_noise):
    """n boxes whose centres lie r_lo..r_hi from `centre` in random
    directions, half extents U(half_lo, half_hi), uniform rotations, stored
    quaternions scaled off unit norm by up to quat_noise."""
    dirs = rng.normal(size=(n, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    c = np.asarray(centre, np.float64) + dirs * rng.uniform(r_lo, r_hi, (n, 1))
    d, p = _pack_many(rng.uniform(half_lo, half_hi, (n, 3)), c, quat_noise, rng)
    return d, p, np.ones(n, np.uint8)


def _rot(qv):
    """Rotation matrices [n, 3, 3] of unit quaternions (w, x, y, z) [n, 4]."""
    w, x, y, z = qv.T
    return np.stack([np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)], -1),
                     np.stack([2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)], -1),
                     np.stack([2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], -1)], 1)


def _pack_many(half, centres, quat_noise, rng):
    """Vectorised pack_obbs (stored pose: q_s = conj(Q), t = -R(q_s) P) with
    the stored quaternions then scaled off unit norm by up to quat_noise."""
    n = len(half)
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    qs = q * np.array([1.0, -1.0, -1.0, -1.0])
    t = -np.einsum("nij,nj->ni", _rot(qs), centres)
    d = np.zeros((n, 4), np.float32)
    d[:, :3] = 2.0 * half
    p = np.zeros((n, 8), np.float32)
    p[:, :3] = t
    p[:, 3:7] = qs * (1.0 + rng.uniform(-quat_noise, quat_noise, (n, 1)))
    return d, p


def _near_surface_spheres(rng, d, p, band):
    """One sphere per box whose surface distance is radius + U(-band, band):
    a point on a face, edge or corner of the (local-frame) box (1, 2 or 3
    saturated axes) pushed out along an outward normal of that region, mapped
    back to the world with the inverse of the stored pose (its quaternion
    normalised)."""
    n = len(d)
    half = d[:, :3].astype(np.float64) * 0.5
    k = rng.choice([1, 2, 3], n, p=[0.6, 0.3, 0.1])
    sat = np.argsort(rng.random((n, 3)), axis=1) < k[:, None]        # which axes are saturated
    sgn = rng.choice([-1.0, 1.0], (n, 3))
    loc = np.where(sat, sgn * half, rng.uniform(-1.0, 1.0, (n, 3)) * half)
    dirs = np.where(sat, sgn * rng.uniform(0.2, 1.0, (n, 3)), 0.0)
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    r = rng.uniform(0.01, 0.1, n)
    loc = loc + dirs * (r + rng.uniform(-band, band, n))[:, None]
    qv = p[:, 3:7].astype(np.float64)
    qv /= np.linalg.norm(qv, axis=1, keepdims=True)
    world = np.einsum("nji,nj->ni", _rot(qv), loc - p[:, :3].astype(np.float64))   # R^T (local - t)
    return np.concatenate([world, r[:, None]], 1).astype(np.float32)


def test_pairs_bitexact_far_large_nonunit():
    """1.2 M pairs, many of them inside the guard band: decisions equal the
    reference's sphere_single_obb_collision and the exact-sequence local
    coordinates equal its transform_sphere_to_local, bit for bit."""
    rng = np.random.default_rng(2024)
    n = 1_200_000
    dirs = rng.normal(size=(n, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    centres = dirs * rng.uniform(5.0, 20.0, (n, 1))
    d, p = _pack_many(rng.uniform(0.02, 2.0, (n, 3)), centres, 1e-3, rng)
    band = (20.0 + 2.0 + 20.0 + 1.0) * 2.0 ** -15
    s = _near_surface_spheres(rng, d, p, 1.5 * band)
    dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (d, p, s)]
    dec = torch.empty(n, dtype=torch.uint8, device="cuda")
    loc = torch.empty((n, 3), dtype=torch.float32, device="cuda")
    _lib.check(_lib.load().ps_debug_obb_pairs(dev[0].data_ptr(), dev[1].data_ptr(), dev[2].data_ptr(), n,
                                              dec.data_ptr(), loc.data_ptr(), None))
    dec = dec.cpu().numpy()
    ref_hit = oracle.ref_obb_pairs(d, p, s)
    ref_loc = oracle.ref_transform_to_local(p, s[:, :3])
    in_band = (dec & 2) != 0
    print(f"pairs: {n}, inside the guard band {in_band.mean():.3f}, hits {(ref_hit != 0).mean():.3f}")
    assert in_band.mean() > 0.05
    assert 0.05 < (ref_hit != 0).mean() < 0.95
    np.testing.assert_array_equal(dec & 1, ref_hit)
    assert np.array_equal(loc.cpu().numpy().view(np.uint32), ref_loc.view(np.uint32))


def _far_robot(offset):
    """The Panda-like chain with its first joint's fixed transform (which
    carries every link) translated by `offset`; the root frame itself is the
    identity in the reference FK."""
    a = workloads.panda_like()
    ft = list(a["fixed_transforms"])
    for k, v in zip((16 + 3, 16 + 7, 16 + 11), offset):
        ft[k] = float(np.float32(ft[k] + v))
    a = dict(a)
    a["fixed_transforms"] = ft
    return a


@pytest.mark.parametrize("offset", [(6.0, -4.0, 3.0), (-11.0, 9.5, 13.0)])
def test_verdicts_bitexact_far_scene(offset):
    """The Panda-like chain based 7-20 m from the origin among 48 boxes 0.4-1.5
    m from its base (full extents up to 1 m) and 4 boxes 2.2-3 m from it
    (full extents up to 2 m), all with non-unit stored quaternions:
    configuration verdicts (also with margins on each configuration's own
    distance to contact) and edge verdicts equal the reference kernels bit
    for bit."""
    rng = np.random.default_rng(77)
    asset = _far_robot(offset)
    small = _shell_boxes(rng, 48, offset, 0.4, 1.5, 0.02, 0.5, 1e-3)
    large = _shell_boxes(rng, 4, offset, 2.2, 3.0, 0.5, 1.0, 1e-3)
    obbs = tuple(np.concatenate([a, b]) for a, b in zip(small, large))
    b = RobotModelBuilder.from_asset(asset).build()
    sc = SceneTensors(*obbs)
    ref = oracle.RefKernels(b, *obbs)
    om = oracle.OracleModel(b, *obbs)
    q = workloads.uniform_configs(rng, asset, 2048)
    hit, _ = api.check_configs(b, sc, torch.from_numpy(q).cuda())
    rhit, _ = ref.check_configs(q)
    np.testing.assert_array_equal(hit.cpu().numpy(), rhit)
    assert 0.05 < rhit.mean() < 0.95
    # near ties: the margin on the FP64 distance to contact, +-1 ulp
    _, _, gap = om.check_configs(q[:64], flags=_lib.PS_NO_GATE)
    n_true = 0
    for i in range(64):
        base = np.float32(gap[i]) if np.isfinite(gap[i]) and abs(gap[i]) < 0.5 else np.float32(0.0)
        for k in (-1, 0, 1):
            m = np.nextafter(base, np.float32(np.inf * k)) if k else base
            one = q[i:i + 1]
            h, _ = api.check_configs(b, sc, torch.from_numpy(one).cuda(), collision_margin=float(m))
            rh, _ = ref.check_configs(one, float(m))
            assert int(h.item()) == int(rh[0]), (i, k, float(m))
            n_true += int(rh[0])
    assert n_true > 0
    frm, to, G = workloads.edge_batch(rng, asset, 3000)
    f, t, g = (torch.from_numpy(x).cuda() for x in (frm, to, G))
    v, c, _ = api.check_edges(b, sc, f, t, samples=g)
    rv, rc, _ = ref.check_edges(frm, to, G)
    np.testing.assert_array_equal(v.cpu().numpy(), rv)
    assert np.array_equal(c.cpu().numpy().view(np.uint32), rc.view(np.uint32))
