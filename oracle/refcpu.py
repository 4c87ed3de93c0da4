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
    ip = C.POINTER(C.c_int32)
    L.nxo_linear_solve.argtypes = [C.c_int32, C.c_int64, ip, ip, dp, dp, dp]
    L.nxo_ipc_step.argtypes = [vp, C.c_double, C.POINTER(abi.NxdIpcParams), C.POINTER(abi.NxdIpcStats)]
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
    i64p = C.POINTER(C.c_int64)
    L.nxo_ipc_candidates.argtypes = [vp, dp, dp, C.c_double, ip, i64, ip, i64, i64p, i64p]
    L.nxo_ipc_barrier.argtypes = [vp, dp, C.c_double, C.c_double, dp, dp, dp, i64p, i64p]
    L.nxo_ipc_max_step.restype = C.c_double
    L.nxo_ipc_max_step.argtypes = [vp, dp, dp, C.c_double, i64p]
    L.nxo_ipc_friction.argtypes = [vp, dp, dp, C.c_double, C.c_double, C.c_double, C.c_double, dp, dp, dp, i64p]
    L.nxo_ipc_friction_derivs.argtypes = [C.c_int32, dp, dp, C.c_double, C.c_double, C.c_double, C.c_double, dp, dp,
                                          dp, C.POINTER(C.c_int32)]
    L.nxo_ipc_pair.argtypes = [C.c_int32, dp, C.c_double, C.c_double, dp, ip, dp, dp, dp, dp, dp]
    L.nxo_ipc_accd.restype = C.c_double
    L.nxo_ipc_accd.argtypes = [C.c_int32, dp, dp, C.c_double, C.c_double, C.c_int32, ip]
    L.nxo_body_count.restype = C.c_int32
    L.nxo_body_count.argtypes = [vp]
    L.nxo_prim_counts.argtypes = [vp, i64p, i64p, i64p]
    L.nxo_prim_topology.argtypes = [vp, ip, ip, ip, ip, ip]
    L.nxo_world_vertices_at.argtypes = [vp, dp, dp, dp]
    L.nxo_ipc_dist2.restype = C.c_double
    L.nxo_ipc_dist2.argtypes = [C.c_int32, dp]
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


    # --- primitive-level contact model (full IPC), ipc_cpu.cpp
    def ipc_candidates(self, x=None, dx=None, inflation: float = 0.0):
        """(pt, ee) int32 arrays of shape (n, 2), sorted."""
        L = lib()
        npt, nee = C.c_int64(), C.c_int64()
        xa = None if x is None else np.ascontiguousarray(x, dtype=np.float64)
        da = None if dx is None else np.ascontiguousarray(dx, dtype=np.float64)
        xp = abi.dptr(xa) if xa is not None else None
        dp_ = abi.dptr(da) if da is not None else None
        L.nxo_ipc_candidates(self.h, xp, dp_, inflation, None, 0, None, 0, C.byref(npt), C.byref(nee))
        pt = np.zeros((max(npt.value, 1), 2), dtype=np.int32)
        ee = np.zeros((max(nee.value, 1), 2), dtype=np.int32)
        L.nxo_ipc_candidates(self.h, xp, dp_, inflation, abi.iptr(pt), npt.value, abi.iptr(ee), nee.value, C.byref(npt),
                             C.byref(nee))
        return pt[:npt.value], ee[:nee.value]

    def ipc_barrier(self, x, dhat: float, kappa: float, hessian: bool = True):
        """(energy, gradient[6N], dense Hessian[6N, 6N] or None, n_pairs, n_active)."""
        n6 = 6 * self.scene.n_bodies
        g = np.zeros(n6)
        H = np.zeros((n6, n6)) if hessian else None
        e = C.c_double()
        npairs, nact = C.c_int64(), C.c_int64()
        lib().nxo_ipc_barrier(self.h, _d(x), dhat, kappa, C.byref(e), abi.dptr(g), abi.dptr(H) if hessian else None,
                              C.byref(npairs), C.byref(nact))
        return e.value, g, H, npairs.value, nact.value

    def ipc_step(self, params=None, dt=None) -> dict:
        """One full-IPC time step (nxo_ipc_step): statistics plus "status"."""
        p = params if params is not None else abi.ipc_params()
        st = abi.NxdIpcStats()
        rc = lib().nxo_ipc_step(self.h, float(self.scene.dt if dt is None else dt), C.byref(p), C.byref(st))
        out = st.as_dict()
        out["status"] = int(rc)
        return out

    def prim_topology(self):
        """(vbody, fbody, fvert [nf, 3], ebody, evert [ne, 2]): the global
        primitive numbering of the full-IPC model (edges in first-seen order
        per body), as the device numbers them."""
        L = lib()
        nv, nf, ne = C.c_int64(), C.c_int64(), C.c_int64()
        L.nxo_prim_counts(self.h, C.byref(nv), C.byref(nf), C.byref(ne))
        vb = np.zeros(max(nv.value, 1), np.int32); fb = np.zeros(max(nf.value, 1), np.int32)
        fv = np.zeros((max(nf.value, 1), 3), np.int32); eb = np.zeros(max(ne.value, 1), np.int32)
        ev = np.zeros((max(ne.value, 1), 2), np.int32)
        L.nxo_prim_topology(self.h, abi.iptr(vb), abi.iptr(fb), abi.iptr(fv), abi.iptr(eb), abi.iptr(ev))
        return vb[:nv.value], fb[:nf.value], fv[:nf.value], eb[:ne.value], ev[:ne.value]

    def world_vertices_at(self, x):
        """(world vertices [nv, 3], body positions [N, 3]) at the iterate x
        (rotations exp(theta) applied to the world's current orientations)."""
        L = lib()
        nv, nf, ne = C.c_int64(), C.c_int64(), C.c_int64()
        L.nxo_prim_counts(self.h, C.byref(nv), C.byref(nf), C.byref(ne))
        wv = np.zeros((max(nv.value, 1), 3))
        pos = np.zeros((self.n, 3))
        L.nxo_world_vertices_at(self.h, _d(x), abi.dptr(wv), abi.dptr(pos))
        return wv[:nv.value], pos

    def ipc_max_step(self, x, dx, eta: float = 0.1):
        n = C.c_int64()
        a = lib().nxo_ipc_max_step(self.h, _d(x), _d(dx), eta, C.byref(n))
        return a, n.value

    def ipc_friction(self, x_lag, x, dhat: float, kappa: float, mu: float, eps: float, hessian: bool = True):
        """Lagged friction alone (nxo_ipc_friction): the pairs active at
        x_lag frozen there, displacements measured from x_lag; (energy,
        gradient[6N], Gauss-Newton Hessian[6N, 6N] or None, frozen pairs) at x."""
        n6 = 6 * self.scene.n_bodies
        g = np.zeros(n6)
        H = np.zeros((n6, n6)) if hessian else None
        e, nf = C.c_double(), C.c_int64()
        lib().nxo_ipc_friction(self.h, _d(x_lag), _d(x), dhat, kappa, mu, eps, C.byref(e), abi.dptr(g),
                               abi.dptr(H) if hessian else None, C.byref(nf))
        return e.value, g, H, nf.value


def ipc_friction_derivs(kind: int, X, Xs, dhat: float, kappa: float, mu: float, eps: float) -> dict:
    """One frozen pair's friction point forces (12) and their derivatives
    with respect to its points (H) and its lag points (Hs), 12 x 12 each
    (ipc::friction_derivs), and the lag points' distance type."""
    X = np.ascontiguousarray(X, dtype=np.float64).reshape(12)
    Xs = np.ascontiguousarray(Xs, dtype=np.float64).reshape(12)
    g, H, Hs = np.zeros(12), np.zeros(144), np.zeros(144)
    t = C.c_int32()
    lib().nxo_ipc_friction_derivs(kind, _d(X), _d(Xs), dhat, kappa, mu, eps, abi.dptr(g), abi.dptr(H), abi.dptr(Hs),
                                  C.byref(t))
    return {"g": g, "H": H.reshape(12, 12), "Hs": Hs.reshape(12, 12), "type": t.value}


def ipc_pair(kind: int, X, dhat: float, kappa: float) -> dict:
    """One pair of four points (kind 0 point-triangle, 1 edge-edge)."""
    X = np.ascontiguousarray(X, dtype=np.float64).reshape(12)
    d2, e = C.c_double(), C.c_double()
    t = C.c_int32()
    g = np.zeros(12)
    Hs, Hr, Hf = np.zeros(144), np.zeros(144), np.zeros(144)
    lib().nxo_ipc_pair(kind, abi.dptr(X), dhat, kappa, C.byref(d2), C.byref(t), C.byref(e), abi.dptr(g), abi.dptr(Hs),
                       abi.dptr(Hr), abi.dptr(Hf))
    return {"d2": d2.value, "type": t.value, "e": e.value, "g": g, "H_sub": Hs.reshape(12, 12),
            "H_raw": Hr.reshape(12, 12), "H_full": Hf.reshape(12, 12)}


def ipc_dist2(kind: int, X) -> float:
    return lib().nxo_ipc_dist2(kind, _d(np.asarray(X, dtype=np.float64).reshape(12)))


def ipc_accd(kind: int, X, D, t_max: float = 1.0, eta: float = 0.1, max_iter: int = 1000):
    it = C.c_int32()
    t = lib().nxo_ipc_accd(kind, _d(np.asarray(X, dtype=np.float64).reshape(12)),
                           _d(np.asarray(D, dtype=np.float64).reshape(12)), t_max, eta, max_iter, C.byref(it))
    return t, it.value


def linear_solve(row_ptr, col_idx, vals, b):
    """LinearSolver restated: x = H^-1 b for a 6x6-block BSR matrix; None on
    a zero pivot."""
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
    col_idx = np.ascontiguousarray(col_idx, dtype=np.int32)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros_like(b)
    ip = C.POINTER(C.c_int32)
    rc = lib().nxo_linear_solve(len(row_ptr) - 1, len(col_idx), row_ptr.ctypes.data_as(ip),
                                col_idx.ctypes.data_as(ip), _d(vals), _d(b), abi.dptr(x))
    return x if rc == 0 else None


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
