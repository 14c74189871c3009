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
