"""ctypes binding of the CPU oracle (oracle/_build/librefcpu.so).

Test infrastructure only: tests/, the smoke check and bench.py's CPU-baseline
leg use it to check or time the reference algorithm.  The product package
never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from nexdynipc_b200 import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "librefcpu.so")
_lib = None


def build() -> str:
    subprocess.check_call([os.path.join(_HERE, "build.sh")])
    return _LIB_PATH


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    L = C.CDLL(_LIB_PATH)
    vp, dp, ip, i64 = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int32), C.c_int64
    L.nxo_create.restype = vp
    L.nxo_create.argtypes = [C.POINTER(abi.NxdSceneDesc)]
    L.nxo_destroy.argtypes = [vp]
    L.nxo_set_options.argtypes = [vp, C.c_int, C.c_int, C.c_int]
    L.nxo_step.argtypes = [vp, C.c_double]
    L.nxo_get_state.argtypes = [vp, C.POINTER(abi.NxdState)]
    L.nxo_set_state.argtypes = [vp, C.POINTER(abi.NxdState)]
    L.nxo_get_diagnostics.argtypes = [vp, C.POINTER(abi.NxdDiagnostics)]
    L.nxo_get_joint_state.argtypes = [vp, dp, dp]
    L.nxo_last_step_times.argtypes = [vp, dp]
    L.nxo_body_pairs.restype = i64
    L.nxo_body_pairs.argtypes = [vp, C.c_double, ip, i64]
    L.nxo_build_candidates.argtypes = [vp, C.c_double, C.POINTER(abi.NxdCandidates)]
    L.nxo_detect_contacts.argtypes = [vp, dp, C.c_void_p, C.c_int32, ip, ip]
    L.nxo_scene_min_distance.restype = C.c_double
    L.nxo_scene_min_distance.argtypes = [vp, C.c_int]
    L.nxo_max_step.restype = C.c_double
    L.nxo_max_step.argtypes = [vp, C.c_double]
    L.nxo_set_form_state.argtypes = [vp, C.c_void_p, C.c_int32, dp, dp, C.c_double]
    L.nxo_form_value.argtypes = [vp, C.c_int32, dp, dp]
    L.nxo_form_gradient.argtypes = [vp, C.c_int32, dp, dp]
    L.nxo_form_hessian_dense.argtypes = [vp, C.c_int32, dp, dp]
    L.nxo_normal_forces.argtypes = [vp, dp, dp, C.c_int32]
    L.nxo_ldlt_solve.argtypes = [dp, C.c_int32, dp, dp]
    L.nxo_select_top_k.argtypes = [dp, C.c_int32, C.c_int32, ip]
    L.nxo_libm.argtypes = [C.c_int32, dp, dp, dp, C.c_int32]
    L.nxo_std_sort.argtypes = [dp, C.c_int32, ip]
    for nm in ("nxo_barrier_value", "nxo_barrier_gradient", "nxo_barrier_hessian"):
        getattr(L, nm).restype = C.c_double
        getattr(L, nm).argtypes = [C.c_double] * 3
    L.nxo_friction_value.restype = C.c_double
    L.nxo_friction_value.argtypes = [dp, C.c_double, C.c_double, C.c_double]
    L.nxo_friction_value_smooth.restype = C.c_double
    L.nxo_friction_value_smooth.argtypes = [dp, C.c_double, C.c_double, C.c_double]
    for nm in ("nxo_friction_gradient", "nxo_friction_hessian", "nxo_friction_gradient_smooth",
               "nxo_friction_hessian_smooth"):
        getattr(L, nm).argtypes = [dp, C.c_double, C.c_double, C.c_double, dp]
    L.nxo_interval_root_poly.restype = C.c_int
    L.nxo_interval_root_poly.argtypes = [dp, C.c_int32, C.c_double, C.c_double, C.c_double, dp, dp]
    _lib = L
    return L


def _d(a):
    return abi.dptr(np.ascontiguousarray(a, dtype=np.float64))


class OracleWorld:
    """The reference's World + IPCSolver, restated on the CPU."""

    def __init__(self, scene, literal_min_distance: bool = False, threads: int = 1, md_stride: int = 1):
        self.scene = scene
        self._desc = scene.desc()
        self.h = lib().nxo_create(C.byref(self._desc))
        if not self.h:
            raise RuntimeError("nxo_create failed")
        lib().nxo_set_options(self.h, int(literal_min_distance), int(md_stride), int(threads))
        self.n = scene.n_bodies

    def close(self):
        if self.h:
            lib().nxo_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_options(self, literal_min_distance=False, md_stride=1, threads=1):
        lib().nxo_set_options(self.h, int(literal_min_distance), int(md_stride), int(threads))

    def step(self, dt=None):
        lib().nxo_step(self.h, float(self.scene.dt if dt is None else dt))

    def state(self) -> dict:
        sb = abi.StateBuffers(self.n)
        v = sb.view()
        lib().nxo_get_state(self.h, C.byref(v))
        return sb.as_dict()

    def set_state(self, st: dict):
        sb = abi.StateBuffers(self.n).load(st)
        v = sb.view()
        lib().nxo_set_state(self.h, C.byref(v))

    def diagnostics(self) -> dict:
        d = abi.NxdDiagnostics()
        lib().nxo_get_diagnostics(self.h, C.byref(d))
        return d.as_dict()

    def joint_state(self):
        nj = len(self.scene.joint_type)
        lam = np.zeros((nj, 6))
        mu = np.zeros(nj)
        lib().nxo_get_joint_state(self.h, abi.dptr(lam), abi.dptr(mu))
        return lam, mu

    def step_times(self):
        t = np.zeros(6)
        lib().nxo_last_step_times(self.h, abi.dptr(t))
        return t

    def body_pairs(self, r: float) -> np.ndarray:
        n = lib().nxo_body_pairs(self.h, r, None, 0)
        out = np.zeros((max(n, 1), 2), dtype=np.int32)
        lib().nxo_body_pairs(self.h, r, abi.iptr(out), n)
        return out[:n]

    def candidates(self, act: float) -> dict:
        c = abi.NxdCandidates()
        lib().nxo_build_candidates(self.h, act, C.byref(c))
        bufs = {"vv": np.zeros((max(c.vv_count, 1), 4), np.int32), "ev": np.zeros((max(c.ev_count, 1), 5), np.int32),
                "ee": np.zeros((max(c.ee_count, 1), 6), np.int32), "fv": np.zeros((max(c.fv_count, 1), 4), np.int32)}
        counts = {"vv": c.vv_count, "ev": c.ev_count, "ee": c.ee_count, "fv": c.fv_count}
        for k, b in bufs.items():
            setattr(c, k, abi.iptr(b))
            setattr(c, k + "_cap", counts[k])
        lib().nxo_build_candidates(self.h, act, C.byref(c))
        return {k: bufs[k][:counts[k]] for k in bufs}

    def detect_contacts(self, x=None):
        cap = 40000
        out = np.zeros(cap, dtype=abi.CONTACT_DTYPE)
        cnt, raw = C.c_int32(0), C.c_int32(0)
        xp = _d(x) if x is not None else None
        lib().nxo_detect_contacts(self.h, xp, out.ctypes.data_as(C.c_void_p), cap, C.byref(cnt), C.byref(raw))
        return out[:cnt.value].copy(), raw.value

    def scene_min_distance(self, literal: bool) -> float:
        return lib().nxo_scene_min_distance(self.h, int(literal))

    def max_step(self, dt: float) -> float:
        return lib().nxo_max_step(self.h, dt)

    def set_form_state(self, contacts, normal_forces=None, x_hat=None, dt=None):
        contacts = np.ascontiguousarray(contacts, dtype=abi.CONTACT_DTYPE)
        nf = _d(normal_forces) if normal_forces is not None else None
        xh = _d(x_hat) if x_hat is not None else None
        self._keep = (contacts, normal_forces, x_hat)
        lib().nxo_set_form_state(self.h, contacts.ctypes.data_as(C.c_void_p), len(contacts), nf, xh,
                                 float(self.scene.dt if dt is None else dt))

    def form_value(self, form: int, x) -> float:
        out = C.c_double(0)
        lib().nxo_form_value(self.h, form, _d(x), C.byref(out))
        return out.value

    def form_gradient(self, form: int, x) -> np.ndarray:
        g = np.zeros(self.n * 6)
        lib().nxo_form_gradient(self.h, form, _d(x), abi.dptr(g))
        return g

    def form_hessian(self, form: int, x) -> np.ndarray:
        H = np.zeros((self.n * 6, self.n * 6))
        lib().nxo_form_hessian_dense(self.h, form, _d(x), abi.dptr(H))
        return H

    def normal_forces(self, x, n) -> np.ndarray:
        out = np.zeros(max(n, 1))
        lib().nxo_normal_forces(self.h, _d(x), abi.dptr(out), n)
        return out[:n]


def libm(fn: int, x, y=None) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(np.zeros_like(x) if y is None else y, dtype=np.float64)
    out = np.zeros_like(x)
    lib().nxo_libm(fn, abi.dptr(x), abi.dptr(y), abi.dptr(out), len(x))
    return out


def select_top_k(scores, k: int) -> np.ndarray:
    s = np.ascontiguousarray(scores, dtype=np.float64)
    out = np.zeros(max(k, 1), dtype=np.int32)
    lib().nxo_select_top_k(abi.dptr(s), len(s), k, abi.iptr(out))
    return out[:min(k, len(s))]


def std_sort(keys, idx=None) -> np.ndarray:
    k = np.ascontiguousarray(keys, dtype=np.float64)
    i = np.arange(len(k), dtype=np.int32) if idx is None else np.ascontiguousarray(idx, dtype=np.int32).copy()
    lib().nxo_std_sort(abi.dptr(k), len(k), abi.iptr(i))
    return i
