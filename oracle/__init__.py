"""Python access to the CPU oracle (liboracle.so) and the reference-kernel
harness (_ref/libref_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference legs, never by the product package.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
ORACLE_LIB = _HERE / "liboracle.so"
REF_LIB = _HERE / "_ref" / "libref_oracle.so"

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)
_u8p = C.POINTER(C.c_uint8)

_lib = None


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def _ptr(a, t):
    return None if a is None else a.ctypes.data_as(t)


def load():
    global _lib
    if _lib is None:
        if not ORACLE_LIB.is_file():
            raise ImportError(f"oracle library missing: {ORACLE_LIB} (make -C oracle)")
        lib = C.CDLL(str(ORACLE_LIB))
        lib.orc_model_create.restype = C.c_void_p
        lib.orc_model_create.argtypes = [C.c_void_p]
        lib.orc_model_destroy.argtypes = [C.c_void_p]
        lib.orc_scene_create.restype = C.c_void_p
        lib.orc_scene_create.argtypes = [_fp, _fp, _u8p, C.c_int, _fp, _fp, _u8p, _fp, C.c_int,
                                         C.c_int, _u8p, _u8p, _u8p, C.c_int]
        lib.orc_scene_destroy.argtypes = [C.c_void_p]
        lib.orc_scene_set_masks.argtypes = [C.c_void_p, _u8p, C.c_int, _u8p, C.c_int, _u8p, C.c_int]
        lib.orc_fk_spheres.argtypes = [C.c_void_p, _fp, C.c_int, C.c_int, _dp]
        lib.orc_check_configs.argtypes = [C.c_void_p, C.c_void_p, _fp, C.c_int, C.c_float, C.c_uint,
                                          C.c_int, C.c_int, _u8p, _dp, _dp]
        lib.orc_check_edges.argtypes = [C.c_void_p, C.c_void_p, _fp, _fp, _ip, C.c_int, C.c_float,
                                        C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _u8p, _dp, _dp,
                                        _dp, C.POINTER(C.c_longlong)]
        lib.orc_state_cost.argtypes = [C.c_void_p, C.c_void_p, _fp, C.c_int, C.c_float, C.c_float,
                                       C.c_float, C.c_int, C.c_int, C.c_int, _dp]
        lib.orc_state_cost_d.restype = C.c_double
        lib.orc_state_cost_d.argtypes = [C.c_void_p, C.c_void_p, _dp, C.c_double, C.c_double,
                                         C.c_double, C.c_int]
        lib.orc_state_cost_kink_distance.restype = C.c_double
        lib.orc_state_cost_kink_distance.argtypes = [C.c_void_p, C.c_void_p, _dp, C.c_double,
                                                     C.c_double, C.c_int]
        lib.orc_state_cost_fd_grad.argtypes = [C.c_void_p, C.c_void_p, _fp, C.c_int, C.c_float,
                                               C.c_float, C.c_float, C.c_int, C.c_double, C.c_int, _dp]
        lib.orc_control_cost_R.argtypes = [C.c_int, C.c_double, _dp]
        _lib = lib
    return _lib


def default_threads() -> int:
    return max(1, len(os.sched_getaffinity(0)))


class OracleModel:
    """CPU oracle over one robot model and one scene (host arrays)."""

    def __init__(self, builder, obb_dims, obb_pose, obb_enable=None, esdf=None, esdf_mode=0):
        lib = load()
        desc, self._keep = builder.descriptor()
        self.n_dof = builder.n_dof
        self.n_spheres = len(builder.sphere_to_joint)
        self.m = lib.orc_model_create(C.byref(desc))
        if not self.m:
            raise ValueError("oracle rejected the model")
        d = _f32(obb_dims).reshape(-1, 4)
        p = _f32(obb_pose).reshape(-1, 8)
        en = (np.ones(len(d), np.uint8) if obb_enable is None
              else np.ascontiguousarray(obb_enable, np.uint8))
        self._scene_keep = [d, p, en]
        if esdf is not None:
            vp, vpose, ven, vfeat = (np.ascontiguousarray(x) for x in esdf)
            vp, vpose, vfeat = _f32(vp), _f32(vpose), _f32(vfeat)
            ven = np.ascontiguousarray(ven, np.uint8)
            self._scene_keep += [vp, vpose, ven, vfeat]
            nl, mv = vp.reshape(-1, 4).shape[0], vfeat.reshape(vp.reshape(-1, 4).shape[0], -1).shape[1]
            self.s = lib.orc_scene_create(_ptr(d, _fp), _ptr(p, _fp), _ptr(en, _u8p), len(d),
                                          _ptr(vp, _fp), _ptr(vpose, _fp), _ptr(ven, _u8p),
                                          _ptr(vfeat, _fp), nl, mv, None, None, None, esdf_mode)
        else:
            self.s = lib.orc_scene_create(_ptr(d, _fp), _ptr(p, _fp), _ptr(en, _u8p), len(d),
                                          None, None, None, None, 0, 0, None, None, None, 0)

    def set_masks(self, acm=None, obb_acm=None, obb_acm_apx=None):
        keep = [None if a is None else np.ascontiguousarray(a, np.uint8).reshape(-1)
                for a in (acm, obb_acm, obb_acm_apx)]
        self._mask_keep = keep
        load().orc_scene_set_masks(self.s, *[x for a in keep for x in
                                             ((_ptr(a, _u8p), 0 if a is None else a.size))])

    def __del__(self):
        try:
            lib = load()
            lib.orc_scene_destroy(self.s)
            lib.orc_model_destroy(self.m)
        except Exception:
            pass

    def fk_spheres(self, q, prec=64):
        q = _f32(q).reshape(-1, self.n_dof)
        out = np.zeros((len(q), self.n_spheres, 3))
        load().orc_fk_spheres(self.m, _ptr(q, _fp), len(q), prec, _ptr(out, _dp))
        return out

    def check_configs(self, q, margin=0.0, flags=0, prec=64, threads=None, want_gap=True):
        q = _f32(q).reshape(-1, self.n_dof)
        n = len(q)
        hit = np.zeros(n, np.uint8)
        clr = np.zeros(n)
        gap = np.zeros(n) if want_gap else None
        load().orc_check_configs(self.m, self.s, _ptr(q, _fp), n, margin, flags, prec,
                                 threads or default_threads(), _ptr(hit, _u8p), _ptr(clr, _dp),
                                 _ptr(gap, _dp))
        return hit, clr, gap

    def check_edges(self, frm, to, G, margin=0.0, check_self=False, compute_clearance=False,
                    early_exit=True, prec=64, threads=None, want_gap=False):
        frm = _f32(frm).reshape(-1, self.n_dof)
        to = _f32(to).reshape(-1, self.n_dof)
        G = np.ascontiguousarray(G, np.int32)
        n = len(frm)
        valid = np.zeros(n, np.uint8)
        cost = np.zeros(n)
        clr = np.zeros(n)
        gap = np.zeros(n) if want_gap else None
        done = C.c_longlong(0)
        load().orc_check_edges(self.m, self.s, _ptr(frm, _fp), _ptr(to, _fp), _ptr(G, _ip), n,
                               margin, int(check_self), int(compute_clearance), int(early_exit),
                               prec, threads or default_threads(), _ptr(valid, _u8p), _ptr(cost, _dp),
                               _ptr(clr, _dp), _ptr(gap, _dp), C.byref(done))
        return valid, cost, clr, gap, done.value

    def state_cost(self, q, w, world_margin, self_margin, include_self=True, prec=64, threads=None):
        q = _f32(q).reshape(-1, self.n_dof)
        out = np.zeros(len(q))
        load().orc_state_cost(self.m, self.s, _ptr(q, _fp), len(q), w, world_margin, self_margin,
                              int(include_self), prec, threads or default_threads(), _ptr(out, _dp))
        return out

    def state_cost_fd_grad(self, q, w, world_margin, self_margin, include_self=True, h=1e-6,
                           threads=None):
        q = _f32(q).reshape(-1, self.n_dof)
        g = np.zeros(q.shape)
        load().orc_state_cost_fd_grad(self.m, self.s, _ptr(q, _fp), len(q), w, world_margin,
                                      self_margin, int(include_self), h, threads or default_threads(),
                                      _ptr(g, _dp))
        return g

    def kink_distance(self, q, world_margin, self_margin, include_self=True):
        q = np.asarray(q, np.float32).reshape(-1, self.n_dof).astype(np.float64)
        out = np.zeros(len(q))
        lib = load()
        for i in range(len(q)):
            row = np.ascontiguousarray(q[i])
            out[i] = lib.orc_state_cost_kink_distance(self.m, self.s, _ptr(row, _dp), world_margin,
                                                      self_margin, int(include_self))
        return out


def control_cost_R(T: int, dt: float) -> np.ndarray:
    R = np.zeros((T, T))
    load().orc_control_cost_R(T, dt, _ptr(R, _dp))
    return R


# ---------------------------------------------------------------------------
# Reference kernels (oracle/_ref/libref_oracle.so, built from the reference
# sources by oracle/Makefile). GPU only.
# ---------------------------------------------------------------------------
_ref = None


def load_ref():
    global _ref
    if _ref is None:
        if not REF_LIB.is_file():
            raise ImportError(f"reference harness missing: {REF_LIB} (make -C oracle ref)")
        lib = C.CDLL(str(REF_LIB))
        lib.ref_model_create.restype = C.c_void_p
        lib.ref_model_create.argtypes = [C.c_void_p]
        lib.ref_model_destroy.argtypes = [C.c_void_p]
        lib.ref_scene_create.restype = C.c_void_p
        lib.ref_scene_create.argtypes = [_fp, _fp, _u8p, C.c_int, _fp, _fp, _u8p, _fp, C.c_int, C.c_int,
                                         _u8p, C.c_int, _u8p, C.c_int, _u8p, C.c_int]
        lib.ref_scene_destroy.argtypes = [C.c_void_p]
        lib.ref_check_configs.argtypes = [C.c_void_p, C.c_void_p, _fp, C.c_int, C.c_float, _u8p, _fp]
        lib.ref_fk_spheres.argtypes = [C.c_void_p, _fp, C.c_int, _fp]
        lib.ref_obb_min_clearance.argtypes = [C.c_void_p, C.c_void_p, _fp, C.c_int, C.c_float, _fp]
        lib.ref_transform_to_local.argtypes = [_fp, _fp, C.c_int, _fp]
        lib.ref_obb_pairs.argtypes = [_fp, _fp, _fp, C.c_int, _u8p]
        lib.ref_check_edges.argtypes = [C.c_void_p, C.c_void_p, _fp, _fp, _ip, C.c_int, C.c_float, C.c_int,
                                        _u8p, _fp, _fp, C.c_int]
        lib.ref_esdf_min_clearance.argtypes = [C.c_void_p, C.c_void_p, _fp, C.c_int, C.c_float, _fp]
        lib.ref_chomp.argtypes = [C.c_void_p, C.c_void_p, _fp, C.c_int, C.c_int, C.c_float, C.c_float,
                                  C.c_float, C.c_float, _fp, _fp, _fp, C.c_int]
        lib.ref_stomp_state_cost.argtypes = [C.c_void_p, C.c_void_p, _fp, C.c_int, C.c_int, C.c_float,
                                             C.c_float, C.c_float, _fp, _fp, C.c_int]
        lib.ref_chomp_solve.argtypes = [C.c_void_p, C.c_void_p, _fp, _fp, C.c_int, C.c_int, C.c_void_p, _fp,
                                        _u8p, _ip, _fp, C.POINTER(C.c_double)]
        lib.ref_stomp_solve.argtypes = [C.c_void_p, C.c_void_p, _fp, _fp, C.c_int, C.c_int, C.c_void_p, _fp,
                                        _u8p, _ip, _fp, C.POINTER(C.c_double)]
        _ref = lib
    return _ref


def _chk(rc, what):
    if rc != 0:
        raise RuntimeError(f"reference harness {what} failed ({rc})")


class RefKernels:
    """PrismPlan's own CUDA kernels on given host inputs (host in, host out)."""

    def __init__(self, builder, obb_dims, obb_pose, obb_enable=None, esdf=None, masks=None):
        lib = load_ref()
        desc, self._keep = builder.descriptor()
        self.n_dof = builder.n_dof
        self.n_spheres = len(builder.sphere_to_joint)
        self.m = lib.ref_model_create(C.byref(desc))
        d = _f32(obb_dims).reshape(-1, 4)
        p = _f32(obb_pose).reshape(-1, 8)
        en = (np.ones(len(d), np.uint8) if obb_enable is None else np.ascontiguousarray(obb_enable, np.uint8))
        keep = [d, p, en]
        vp = vpose = ven = vfeat = None
        nl = mv = 0
        if esdf is not None:
            vp, vpose, ven, vfeat = (np.ascontiguousarray(x) for x in esdf)
            vp, vpose, vfeat = _f32(vp), _f32(vpose), _f32(vfeat)
            ven = np.ascontiguousarray(ven, np.uint8)
            nl = vp.reshape(-1, 4).shape[0]
            mv = vfeat.reshape(nl, -1).shape[1]
            keep += [vp, vpose, ven, vfeat]
        m = masks or {}
        mk = [None if m.get(k) is None else np.ascontiguousarray(m[k], np.uint8).reshape(-1)
              for k in ("acm", "obb_acm", "obb_acm_apx")]
        keep += mk
        self._scene_keep = keep
        self.s = lib.ref_scene_create(_ptr(d, _fp), _ptr(p, _fp), _ptr(en, _u8p), len(d), _ptr(vp, _fp),
                                      _ptr(vpose, _fp), _ptr(ven, _u8p), _ptr(vfeat, _fp), nl, mv,
                                      _ptr(mk[0], _u8p), 0 if mk[0] is None else mk[0].size,
                                      _ptr(mk[1], _u8p), 0 if mk[1] is None else mk[1].size,
                                      _ptr(mk[2], _u8p), 0 if mk[2] is None else mk[2].size)

    def __del__(self):
        try:
            lib = load_ref()
            lib.ref_scene_destroy(self.s)
            lib.ref_model_destroy(self.m)
        except Exception:
            pass

    def check_configs(self, q, margin=0.0):
        q = _f32(q).reshape(-1, self.n_dof)
        hit = np.zeros(len(q), np.uint8)
        ms = C.c_float(0)
        _chk(load_ref().ref_check_configs(self.m, self.s, _ptr(q, _fp), len(q), margin, _ptr(hit, _u8p),
                                          C.byref(ms)), "check_configs")
        return hit, ms.value

    def fk_spheres(self, q):
        q = _f32(q).reshape(-1, self.n_dof)
        out = np.zeros((len(q), self.n_spheres, 3), np.float32)
        _chk(load_ref().ref_fk_spheres(self.m, _ptr(q, _fp), len(q), _ptr(out, _fp)), "fk")
        return out

    def obb_min_clearance(self, q, margin=0.0):
        q = _f32(q).reshape(-1, self.n_dof)
        out = np.zeros(len(q), np.float32)
        _chk(load_ref().ref_obb_min_clearance(self.m, self.s, _ptr(q, _fp), len(q), margin, _ptr(out, _fp)),
             "obb_min_clearance")
        return out

    def esdf_min_clearance(self, q, margin=0.0):
        """scene_min_clearance_runtime per configuration (4-thread blocks)."""
        q = _f32(q).reshape(-1, self.n_dof)
        out = np.zeros(len(q), np.float32)
        _chk(load_ref().ref_esdf_min_clearance(self.m, self.s, _ptr(q, _fp), len(q), margin, _ptr(out, _fp)),
             "esdf_min_clearance")
        return out

    def check_edges(self, frm, to, G, margin=0.0, check_self=False, reps=1):
        frm = _f32(frm).reshape(-1, self.n_dof)
        to = _f32(to).reshape(-1, self.n_dof)
        G = np.ascontiguousarray(G, np.int32)
        valid = np.zeros(len(frm), np.uint8)
        cost = np.zeros(len(frm), np.float32)
        ms = C.c_float(0)
        _chk(load_ref().ref_check_edges(self.m, self.s, _ptr(frm, _fp), _ptr(to, _fp), _ptr(G, _ip), len(frm),
                                        margin, int(check_self), _ptr(valid, _u8p), _ptr(cost, _fp), C.byref(ms),
                                        reps), "edges")
        return valid, cost, ms.value

    def chomp(self, theta_bdt, w, world_margin, self_margin, fd_eps=1e-3, state=True, grad=True, reps=1):
        th = _f32(theta_bdt)
        B, D, T = th.shape
        sc = np.zeros_like(th) if state else None
        g = np.zeros_like(th) if grad else None
        ms = C.c_float(0)
        _chk(load_ref().ref_chomp(self.m, self.s, _ptr(th, _fp), B, T, w, world_margin, self_margin, fd_eps,
                                  _ptr(sc, _fp), _ptr(g, _fp), C.byref(ms), reps), "chomp")
        return sc, g, ms.value

    def chomp_solve(self, starts, goals, T, params):
        """CHOMP::solve_runtime_scene per request (chomp.cu:358-600).
        params: a ps_chomp_params ctypes structure. Returns (path [B,T,D],
        solved [B] u8, iterations [B] i32, final_total_cost [B], wall ms)."""
        return self._solve(load_ref().ref_chomp_solve, starts, goals, T, params, "chomp_solve")

    def stomp_solve(self, starts, goals, T, params):
        """STOMP::solve_runtime_scene per request (stomp.cu:565-965), with a
        ps_stomp_params structure; outputs as chomp_solve."""
        return self._solve(load_ref().ref_stomp_solve, starts, goals, T, params, "stomp_solve")

    def _solve(self, fn, starts, goals, T, params, what):
        st = _f32(starts).reshape(-1, self.n_dof)
        gl = _f32(goals).reshape(-1, self.n_dof)
        B = len(st)
        path = np.zeros((B, T, self.n_dof), np.float32)
        solved = np.zeros(B, np.uint8)
        iters = np.zeros(B, np.int32)
        total = np.zeros(B, np.float32)
        ms = C.c_double(0)
        _chk(fn(self.m, self.s, _ptr(st, _fp), _ptr(gl, _fp), B, int(T), C.byref(params), _ptr(path, _fp),
                _ptr(solved, _u8p), _ptr(iters, _ip), _ptr(total, _fp), C.byref(ms)), what)
        return path, solved, iters, total, ms.value

    def stomp(self, rollouts_bdt, w, world_margin, self_margin, reps=1):
        r = _f32(rollouts_bdt)
        R, D, T = r.shape
        out = np.zeros_like(r)
        ms = C.c_float(0)
        _chk(load_ref().ref_stomp_state_cost(self.m, self.s, _ptr(r, _fp), R, T, w, world_margin, self_margin,
                                             _ptr(out, _fp), C.byref(ms), reps), "stomp")
        return out, ms.value


def ref_transform_to_local(pose, pts):
    pose = _f32(pose).reshape(-1, 8)
    pts = _f32(pts).reshape(-1, 3)
    out = np.zeros_like(pts)
    _chk(load_ref().ref_transform_to_local(_ptr(pose, _fp), _ptr(pts, _fp), len(pts), _ptr(out, _fp)), "to_local")
    return out


def ref_obb_pairs(dims, pose, spheres):
    dims = _f32(dims).reshape(-1, 4)
    pose = _f32(pose).reshape(-1, 8)
    spheres = _f32(spheres).reshape(-1, 4)
    out = np.zeros(len(spheres), np.uint8)
    _chk(load_ref().ref_obb_pairs(_ptr(dims, _fp), _ptr(pose, _fp), _ptr(spheres, _fp), len(spheres),
                                  _ptr(out, _u8p)), "obb_pairs")
    return out
