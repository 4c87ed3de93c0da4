"""Python binding of libnxd_b200.so (the C ABI in include/nxd.h).

`Context` owns one device-resident scene and drives the B200 contact step.
`IPCSolver` / `World` mirror the reference's class names and setters
(nexdynipc/NexDynIPC/Dynamics/IPCSolver.h:21-91) for callers that think in
those terms.  There is no CPU path here: loading fails loudly when the CUDA
library is absent, and every call goes through the shared library.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libnxd_b200.so")
_lib = None


class NxdError(RuntimeError):
    def __init__(self, fn: str, status: int):
        super().__init__(f"{fn} failed: {abi.STATUS_NAMES.get(status, status)}")
        self.status = status


def lib():
    """Load libnxd_b200.so (build it with nexdynipc_b200/build.py)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: run `python nexdynipc_b200/build.py` (no CPU fallback exists)")
    L = C.CDLL(LIB_PATH)
    vp, dp, ip, i64p = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int32), C.POINTER(C.c_int64)
    L.nxd_version.restype = C.c_char_p
    L.nxd_default_settings.argtypes = [C.POINTER(abi.NxdSettings)]
    L.nxd_create.argtypes = [C.POINTER(abi.NxdSceneDesc), C.POINTER(vp)]
    L.nxd_destroy.argtypes = [vp]
    L.nxd_set_stream.argtypes = [vp, vp]
    L.nxd_step.argtypes = [vp, C.c_double]
    L.nxd_get_state.argtypes = [vp, C.POINTER(abi.NxdState)]
    L.nxd_set_state.argtypes = [vp, C.POINTER(abi.NxdState)]
    L.nxd_get_diagnostics.argtypes = [vp, C.POINTER(abi.NxdDiagnostics)]
    L.nxd_get_joint_state.argtypes = [vp, dp, dp]
    L.nxd_body_pairs.argtypes = [vp, C.c_double, ip, C.c_int64, i64p]
    L.nxd_build_candidates.argtypes = [vp, C.c_double, C.POINTER(abi.NxdCandidates)]
    L.nxd_detect_contacts.argtypes = [vp, dp, C.c_void_p, C.c_int32, ip]
    L.nxd_scene_min_distance.argtypes = [vp, dp]
    L.nxd_max_step.argtypes = [vp, C.c_double, dp]
    L.nxd_set_form_state.argtypes = [vp, C.c_void_p, C.c_int32, dp, dp, C.c_double]
    L.nxd_form_value.argtypes = [vp, C.c_int32, dp, dp]
    L.nxd_form_gradient.argtypes = [vp, C.c_int32, dp, dp]
    L.nxd_form_hessian_bsr.argtypes = [vp, C.c_int32, dp, ip, ip, dp, C.c_int64, i64p]
    L.nxd_normal_forces.argtypes = [vp, dp, dp, C.c_int32]
    L.nxd_eval_all.argtypes = [vp, dp, dp, dp, ip, ip, dp, C.c_int64, i64p]
    L.nxd_linear_solve.argtypes = [vp, C.POINTER(abi.NxdBsr), dp, dp, C.POINTER(abi.NxdSolveStats)]
    L.nxd_ipc_step.argtypes = [vp, C.c_double, C.POINTER(abi.NxdIpcParams), C.POINTER(abi.NxdIpcStats)]
    L.nxd_pcg_solve.argtypes = [vp, C.POINTER(abi.NxdBsr), dp, dp, C.c_double, C.c_int32, C.POINTER(abi.NxdPcgStats)]
    L.nxd_batch_create.argtypes = [C.POINTER(abi.NxdSceneDesc), C.c_int32, C.POINTER(vp)]
    L.nxd_batch_destroy.argtypes = [vp]
    L.nxd_batch_step.argtypes = [vp, dp]
    L.nxd_batch_get_state.argtypes = [vp, C.c_int32, C.POINTER(abi.NxdState)]
    L.nxd_batch_get_diagnostics.argtypes = [vp, C.c_int32, C.POINTER(abi.NxdDiagnostics)]
    L.nxd_ipc_candidates.argtypes = [vp, vp, vp, C.c_double, ip, C.c_int64, ip, C.c_int64, i64p, i64p]
    L.nxd_ipc_candidates.restype = C.c_int
    L.nxd_ipc_barrier.argtypes = [vp, vp, C.c_double, C.c_double, dp, dp, ip, ip, dp, C.c_int64, i64p, i64p, i64p]
    L.nxd_ipc_barrier.restype = C.c_int
    L.nxd_ipc_max_step.argtypes = [vp, vp, vp, C.c_double, dp, i64p]
    L.nxd_ipc_max_step.restype = C.c_int
    L.nxd_batch_groups.argtypes = [vp]
    L.nxd_batch_groups.restype = C.c_int32
    L.nxd_batch_set_stream.argtypes = [vp, vp]
    L.nxd_batch_set_stream.restype = C.c_int
    L.nxd_batch_set_queue_ctas.argtypes = [vp, C.c_int32, C.c_int32]
    L.nxd_batch_set_queue_ctas.restype = C.c_int
    L.nxd_batch_timed_steps.argtypes = [vp, dp, C.c_int32, dp]
    L.nxd_batch_timed_steps.restype = C.c_int
    L.nxd_device_info.argtypes = [C.POINTER(C.c_int32), C.c_char_p, C.c_int32]
    L.nxd_device_info.restype = C.c_int
    L.nxd_body_pairs_noalloc.argtypes = [vp, vp, vp, C.c_int32, C.c_double, vp, C.c_int64, i64p, vp]
    L.nxd_body_pairs_noalloc.restype = C.c_int
    L.nxd_ipc_adjoint.argtypes = [vp, C.c_double, C.POINTER(abi.NxdIpcParams), C.POINTER(abi.NxdState), dp, dp,
                                  C.POINTER(abi.NxdIpcAdjointOut)]
    L.nxd_ipc_adjoint.restype = C.c_int
    L.nxd_debug_grid_wait.argtypes = [vp, C.c_uint32, C.c_int32]
    L.nxd_debug_grid_wait.restype = C.c_int
    L.nxd_fp64_peak.argtypes = [vp, dp, dp]
    L.nxd_fp64_peak.restype = C.c_int
    L.nxd_profile.argtypes = [vp, C.c_int32, dp, i64p]
    L.nxd_profile.restype = C.c_int
    for name in ("nxd_set_form_state", "nxd_form_value", "nxd_form_gradient", "nxd_form_hessian_bsr",
                 "nxd_normal_forces", "nxd_batch_create", "nxd_batch_step", "nxd_batch_get_state",
                 "nxd_batch_get_diagnostics"):
        getattr(L, name).restype = C.c_int
    for name in ("nxd_create", "nxd_set_stream", "nxd_step", "nxd_get_state", "nxd_set_state", "nxd_get_diagnostics",
                 "nxd_get_joint_state", "nxd_body_pairs", "nxd_build_candidates", "nxd_detect_contacts",
                 "nxd_scene_min_distance", "nxd_max_step"):
        getattr(L, name).restype = C.c_int
    _lib = L
    return L


def _check(fn: str, st: int):
    if st != 0:
        raise NxdError(fn, st)


class Context:
    """One scene resident on the GPU (World + IPCSolver of the reference)."""

    def __init__(self, scene):
        self.scene = scene
        self._desc = scene.desc()
        h = C.c_void_p()
        _check("nxd_create", lib().nxd_create(C.byref(self._desc), C.byref(h)))
        self.h = h
        self.n = scene.n_bodies

    def close(self):
        if getattr(self, "h", None):
            lib().nxd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, dt=None, n: int = 1):
        dt = float(self.scene.dt if dt is None else dt)
        for _ in range(n):
            _check("nxd_step", lib().nxd_step(self.h, dt))

    def state(self) -> dict:
        sb = abi.StateBuffers(self.n)
        v = sb.view()
        _check("nxd_get_state", lib().nxd_get_state(self.h, C.byref(v)))
        return sb.as_dict()

    def set_state(self, st: dict):
        sb = abi.StateBuffers(self.n).load(st)
        v = sb.view()
        _check("nxd_set_state", lib().nxd_set_state(self.h, C.byref(v)))

    def diagnostics(self) -> dict:
        d = abi.NxdDiagnostics()
        _check("nxd_get_diagnostics", lib().nxd_get_diagnostics(self.h, C.byref(d)))
        return d.as_dict()

    def joint_state(self):
        nj = len(self.scene.joint_type)
        lam = np.zeros((max(nj, 1), 6))
        mu = np.zeros(max(nj, 1))
        _check("nxd_get_joint_state", lib().nxd_get_joint_state(self.h, abi.dptr(lam), abi.dptr(mu)))
        return lam[:nj], mu[:nj]

    def debug_grid_wait(self, spin_limit: int, hold_last_cta: bool):
        """nxd_debug_grid_wait: bound the Newton solve's barrier waits and
        optionally hold its last CTA back (failure-detection tests);
        (0, False) restores the normal solve and clears the sticky status."""
        _check("nxd_debug_grid_wait", lib().nxd_debug_grid_wait(self.h, int(spin_limit), int(hold_last_cta)))

    def body_pairs(self, r: float) -> np.ndarray:
        cnt = C.c_int64(0)
        _check("nxd_body_pairs", lib().nxd_body_pairs(self.h, r, None, 0, C.byref(cnt)))
        out = np.zeros((max(cnt.value, 1), 2), dtype=np.int32)
        _check("nxd_body_pairs", lib().nxd_body_pairs(self.h, r, abi.iptr(out), cnt.value, C.byref(cnt)))
        return out[:cnt.value]

    def candidates(self, act: float) -> dict:
        c = abi.NxdCandidates()
        _check("nxd_build_candidates", lib().nxd_build_candidates(self.h, act, C.byref(c)))
        counts = {"vv": c.vv_count, "ev": c.ev_count, "ee": c.ee_count, "fv": c.fv_count}
        widths = {"vv": 4, "ev": 5, "ee": 6, "fv": 4}
        bufs = {k: np.zeros((max(counts[k], 1), widths[k]), np.int32) for k in counts}
        for k, b in bufs.items():
            setattr(c, k, abi.iptr(b))
            setattr(c, k + "_cap", counts[k])
        _check("nxd_build_candidates", lib().nxd_build_candidates(self.h, act, C.byref(c)))
        return {k: bufs[k][:counts[k]] for k in bufs}

    def candidate_counts(self, act: float):
        """(face-vertex, edge-edge) candidate counts at the current poses."""
        c = abi.NxdCandidates()
        _check("nxd_build_candidates", lib().nxd_build_candidates(self.h, act, C.byref(c)))
        return int(c.fv_count), int(c.ee_count)

    def profile(self, enable: bool):
        """Per-family device milliseconds and launch counts since the last call."""
        ms = np.zeros(9)
        n = np.zeros(9, dtype=np.int64)
        _check("nxd_profile", lib().nxd_profile(self.h, int(enable), abi.dptr(ms),
                                                n.ctypes.data_as(C.POINTER(C.c_int64))))
        return ms, n

    def detect_contacts(self, x=None) -> np.ndarray:
        cap = 40000
        out = np.zeros(cap, dtype=abi.CONTACT_DTYPE)
        cnt = C.c_int32(0)
        xp = abi.dptr(np.ascontiguousarray(x, dtype=np.float64)) if x is not None else None
        _check("nxd_detect_contacts", lib().nxd_detect_contacts(self.h, xp, out.ctypes.data_as(C.c_void_p), cap,
                                                                C.byref(cnt)))
        return out[:cnt.value].copy()

    def scene_min_distance(self) -> float:
        v = C.c_double(0)
        _check("nxd_scene_min_distance", lib().nxd_scene_min_distance(self.h, C.byref(v)))
        return v.value

    def max_step(self, dt: float) -> float:
        v = C.c_double(0)
        _check("nxd_max_step", lib().nxd_max_step(self.h, dt, C.byref(v)))
        return v.value


    # Form plugin interface (Dynamics/Forms/Form.h:8-21)
    def set_form_state(self, contacts, normal_forces=None, x_hat=None, dt=None):
        contacts = np.ascontiguousarray(contacts, dtype=abi.CONTACT_DTYPE)
        self._fs = (contacts, None if normal_forces is None else np.ascontiguousarray(normal_forces, np.float64),
                    None if x_hat is None else np.ascontiguousarray(x_hat, np.float64))
        nf = abi.dptr(self._fs[1]) if normal_forces is not None else None
        xh = abi.dptr(self._fs[2]) if x_hat is not None else None
        _check("nxd_set_form_state", lib().nxd_set_form_state(self.h, contacts.ctypes.data_as(C.c_void_p), len(contacts),
                                                              nf, xh, float(self.scene.dt if dt is None else dt)))

    def form_value(self, form: int, x) -> float:
        v = C.c_double(0)
        _check("nxd_form_value", lib().nxd_form_value(self.h, form, abi.dptr(np.ascontiguousarray(x, np.float64)),
                                                      C.byref(v)))
        return v.value

    def form_gradient(self, form: int, x) -> np.ndarray:
        g = np.zeros(6 * self.n)
        _check("nxd_form_gradient", lib().nxd_form_gradient(self.h, form, abi.dptr(np.ascontiguousarray(x, np.float64)),
                                                            abi.dptr(g)))
        return g

    def form_hessian_bsr(self, x):
        xx = np.ascontiguousarray(x, np.float64)
        nnzb = C.c_int64(0)
        rp = np.zeros(self.n + 1, np.int32)
        st = lib().nxd_form_hessian_bsr(self.h, abi.NXD_FORM_TOTAL, abi.dptr(xx), abi.iptr(rp), None, None, 0,
                                        C.byref(nnzb))
        cap = nnzb.value
        ci = np.zeros(max(cap, 1), np.int32)
        vals = np.zeros((max(cap, 1), 6, 6))
        _check("nxd_form_hessian_bsr", lib().nxd_form_hessian_bsr(self.h, abi.NXD_FORM_TOTAL, abi.dptr(xx), abi.iptr(rp),
                                                                  abi.iptr(ci), abi.dptr(vals), cap, C.byref(nnzb)))
        return rp, ci[:cap], vals[:cap]

    def form_hessian_dense(self, x) -> np.ndarray:
        rp, ci, vals = self.form_hessian_bsr(x)
        H = np.zeros((6 * self.n, 6 * self.n))
        for i in range(self.n):
            for q in range(rp[i], rp[i + 1]):
                j = ci[q]
                H[6 * i:6 * i + 6, 6 * j:6 * j + 6] += vals[q]
        return H

    def eval_all(self, x):
        """(energy, gradient, (row_ptr, col_idx, vals)) of the total energy at
        x in one call (nxd_eval_all)."""
        xx = np.ascontiguousarray(x, np.float64)
        e = C.c_double(0)
        g = np.zeros(6 * self.n)
        rp = np.zeros(self.n + 1, np.int32)
        # every row: its diagonal block plus one block per incident coupling
        # term (joints, control forms, at most 2000 contacts twice)
        cap = self.n + 2 * (len(self.scene.joint_type) + len(self.scene.drive_body_b) + 2 * 2000)
        nnzb = C.c_int64(0)
        ci = np.zeros(cap, np.int32)
        vals = np.zeros((cap, 6, 6))
        _check("nxd_eval_all", lib().nxd_eval_all(self.h, abi.dptr(xx), C.byref(e), abi.dptr(g), abi.iptr(rp),
                                                  abi.iptr(ci), abi.dptr(vals), cap, C.byref(nnzb)))
        return e.value, g, (rp, ci[:nnzb.value], vals[:nnzb.value])

    def linear_solve(self, row_ptr, col_idx, vals, b):
        """x = H^-1 b for a 6x6-block BSR H over this context's bodies
        (nxd_linear_solve); returns (x, stats dict)."""
        rp = np.ascontiguousarray(row_ptr, np.int32)
        ci = np.ascontiguousarray(col_idx, np.int32)
        vv = np.ascontiguousarray(vals, np.float64)
        bb = np.ascontiguousarray(b, np.float64)
        H = abi.NxdBsr(self.n, len(ci), abi.iptr(rp), abi.iptr(ci), abi.dptr(vv))
        x = np.zeros(6 * self.n)
        stt = abi.NxdSolveStats()
        _check("nxd_linear_solve", lib().nxd_linear_solve(self.h, C.byref(H), abi.dptr(bb), abi.dptr(x), C.byref(stt)))
        return x, {k: getattr(stt, k) for k, _ in abi.NxdSolveStats._fields_}

    def pcg_solve(self, row_ptr, col_idx, vals, b, tol: float = 1e-12, max_iter: int = 1000, check: bool = True):
        """x ~ H^-1 b by block-Jacobi PCG (nxd_pcg_solve); returns (x, stats
        dict with the call's status).  H's block rows need not be this
        context's bodies."""
        rp = np.ascontiguousarray(row_ptr, np.int32)
        ci = np.ascontiguousarray(col_idx, np.int32)
        vv = np.ascontiguousarray(vals, np.float64)
        bb = np.ascontiguousarray(b, np.float64)
        H = abi.NxdBsr(len(rp) - 1, len(ci), abi.iptr(rp), abi.iptr(ci), abi.dptr(vv))
        x = np.zeros(len(bb))
        st = abi.NxdPcgStats()
        rc = lib().nxd_pcg_solve(self.h, C.byref(H), abi.dptr(bb), abi.dptr(x), float(tol), int(max_iter), C.byref(st))
        if check and rc not in (0, 1):
            _check("nxd_pcg_solve", rc)
        out = {k: getattr(st, k) for k, _ in abi.NxdPcgStats._fields_}
        out["rc"] = int(rc)
        return x, out

    def normal_forces(self, x, n: int) -> np.ndarray:
        out = np.zeros(max(n, 1))
        _check("nxd_normal_forces", lib().nxd_normal_forces(self.h, abi.dptr(np.ascontiguousarray(x, np.float64)),
                                                            abi.dptr(out), n))
        return out[:n]


    # --- primitive-level contact model (full IPC): nxd_ipc_*
    def ipc_candidates(self, x=None, dx=None, inflation: float = 0.0):
        """Point-triangle (vertex, face) and edge-edge (edge, edge) pairs,
        int32 arrays of shape (n, 2), sorted (LBVH on the device)."""
        L = lib()
        npt, nee = C.c_int64(), C.c_int64()
        xa = None if x is None else np.ascontiguousarray(x, dtype=np.float64)
        da = None if dx is None else np.ascontiguousarray(dx, dtype=np.float64)
        xp = C.c_void_p(xa.ctypes.data) if xa is not None else None
        dp_ = C.c_void_p(da.ctypes.data) if da is not None else None
        _check("nxd_ipc_candidates", L.nxd_ipc_candidates(self.h, xp, dp_, inflation, None, 0, None, 0, C.byref(npt),
                                                          C.byref(nee)))
        pt = np.zeros((max(npt.value, 1), 2), dtype=np.int32)
        ee = np.zeros((max(nee.value, 1), 2), dtype=np.int32)
        _check("nxd_ipc_candidates", L.nxd_ipc_candidates(self.h, xp, dp_, inflation, abi.iptr(pt), npt.value,
                                                          abi.iptr(ee), nee.value, C.byref(npt), C.byref(nee)))
        return pt[:npt.value], ee[:nee.value]

    def ipc_barrier(self, x, dhat: float, kappa: float):
        """(energy, gradient[6N], (row_ptr, col_idx, vals[nnzb, 6, 6]), n_pairs, n_active)."""
        L = lib()
        n = self.scene.n_bodies
        xa = np.ascontiguousarray(x, dtype=np.float64)
        e = C.c_double()
        g = np.zeros(6 * n)
        nnzb, npairs, nact = C.c_int64(), C.c_int64(), C.c_int64()
        rp = np.zeros(n + 1, dtype=np.int32)
        _check("nxd_ipc_barrier", L.nxd_ipc_barrier(self.h, C.c_void_p(xa.ctypes.data), dhat, kappa, C.byref(e), abi.dptr(g),
                                                    abi.iptr(rp), None, None, 0, C.byref(nnzb), C.byref(npairs),
                                                    C.byref(nact)))
        ci = np.zeros(max(nnzb.value, 1), dtype=np.int32)
        vv = np.zeros((max(nnzb.value, 1), 6, 6))
        _check("nxd_ipc_barrier", L.nxd_ipc_barrier(self.h, C.c_void_p(xa.ctypes.data), dhat, kappa, C.byref(e), abi.dptr(g),
                                                    abi.iptr(rp), abi.iptr(ci), abi.dptr(vv), nnzb.value, C.byref(nnzb),
                                                    C.byref(npairs), C.byref(nact)))
        m = nnzb.value
        return e.value, g, (rp, ci[:m], vv[:m]), npairs.value, nact.value

    def ipc_step(self, params=None, dt=None) -> dict:
        """One full-IPC time step (nxd_ipc_step); returns its statistics."""
        p = params if params is not None else abi.ipc_params()
        st = abi.NxdIpcStats()
        _check("nxd_ipc_step", lib().nxd_ipc_step(self.h, float(self.scene.dt if dt is None else dt), C.byref(p),
                                                  C.byref(st)))
        return st.as_dict()

    def ipc_adjoint(self, start: dict, x_star, x_bar, params=None, dt=None) -> dict:
        """nxd_ipc_adjoint: the adjoint of one full-IPC step from the state
        `start` at its converged iterate x_star (6N) for x_bar = dL/dx_star.
        Returns lam (6N), phat_bar / thetahat_bar / phi_bar (N, 3), mass_bar
        (N), inertia_bar (N, 3, 3), joint_mu_bar (J), n_active and, with
        friction (params.mu > 0, one lagging pass), p0_bar (N, 3) and
        friction_mu_bar."""
        n, nj = self.scene.n_bodies, len(self.scene.joint_type)
        p = params if params is not None else abi.ipc_params()
        sb = abi.StateBuffers(n).load(start)
        view = sb.view()
        xs = np.ascontiguousarray(x_star, dtype=np.float64)
        xb = np.ascontiguousarray(x_bar, dtype=np.float64)
        out = {"lam": np.zeros(6 * n), "phat_bar": np.zeros((n, 3)), "thetahat_bar": np.zeros((n, 3)),
               "phi_bar": np.zeros((n, 3)), "mass_bar": np.zeros(n), "inertia_bar": np.zeros((n, 3, 3)),
               "joint_mu_bar": np.zeros(max(nj, 1)), "p0_bar": np.zeros((n, 3)), "friction_mu_bar": np.zeros(1)}
        na = C.c_int32(0)
        o = abi.NxdIpcAdjointOut(*[abi.dptr(out[k]) for k in ("lam", "phat_bar", "thetahat_bar", "phi_bar", "mass_bar",
                                                                "inertia_bar", "joint_mu_bar")], C.pointer(na),
                                 abi.dptr(out["p0_bar"]), abi.dptr(out["friction_mu_bar"]))
        _check("nxd_ipc_adjoint", lib().nxd_ipc_adjoint(self.h, float(self.scene.dt if dt is None else dt), C.byref(p),
                                                        C.byref(view), abi.dptr(xs), abi.dptr(xb), C.byref(o)))
        out["joint_mu_bar"] = out["joint_mu_bar"][:nj]
        out["friction_mu_bar"] = float(out["friction_mu_bar"][0])
        out["n_active"] = na.value
        return out

    def ipc_max_step(self, x, dx, eta: float = 0.1):
        """(alpha, n_pairs): additive-CCD bound of the step x -> x + dx."""
        a = C.c_double()
        n = C.c_int64()
        xa = np.ascontiguousarray(x, dtype=np.float64)
        da = np.ascontiguousarray(dx, dtype=np.float64)
        _check("nxd_ipc_max_step", lib().nxd_ipc_max_step(self.h, C.c_void_p(xa.ctypes.data), C.c_void_p(da.ctypes.data),
                                                          eta, C.byref(a), C.byref(n)))
        return a.value, n.value


QUEUE_KERNELS = {"narrow_rows": 0, "narrow_emit": 1}     # NXD_QUEUE_NARROW_ROWS / _EMIT
AUTOTUNE_CTAS = (1, 2, 4, 8, 16)


def device_info():
    """(SM count, device name) of the current device (nxd_device_info)."""
    sm = C.c_int32()
    buf = C.create_string_buffer(256)
    _check("nxd_device_info", lib().nxd_device_info(C.byref(sm), buf, 256))
    return sm.value, buf.value.decode()


class Batch:
    """Independent scenes stepped together (nxd_batch_*)."""

    def __init__(self, scene_list):
        self.scenes = list(scene_list)
        self._descs = (abi.NxdSceneDesc * len(self.scenes))()
        for i, s in enumerate(self.scenes):
            self._descs[i] = s.desc()
        h = C.c_void_p()
        _check("nxd_batch_create", lib().nxd_batch_create(self._descs, len(self.scenes), C.byref(h)))
        self.h = h
        self.dts = np.array([s.dt for s in self.scenes], dtype=np.float64)

    def close(self):
        if getattr(self, "h", None):
            lib().nxd_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n: int = 1):
        for _ in range(n):
            _check("nxd_batch_step", lib().nxd_batch_step(self.h, abi.dptr(self.dts)))

    def set_stream(self, stream_ptr: int):
        """Issue the batch's work on a caller's CUDA stream (raw cudaStream_t)."""
        _check("nxd_batch_set_stream", lib().nxd_batch_set_stream(self.h, C.c_void_p(stream_ptr)))

    def groups(self) -> int:
        """Number of launch groups (scenes with identical step sequences)."""
        return int(lib().nxd_batch_groups(self.h))

    def set_queue_ctas(self, kernel: int, ctas_per_sm: int):
        """Persistent grid (CTAs per SM) of a queue-form narrow-phase kernel
        (QUEUE_NARROW_ROWS / QUEUE_NARROW_EMIT); results do not depend on it."""
        _check("nxd_batch_set_queue_ctas", lib().nxd_batch_set_queue_ctas(self.h, int(kernel), int(ctas_per_sm)))

    def timed_steps(self, n: int) -> float:
        """n steps timed by CUDA events on the batch's stream; milliseconds."""
        ms = C.c_double()
        _check("nxd_batch_timed_steps", lib().nxd_batch_timed_steps(self.h, abi.dptr(self.dts), int(n), C.byref(ms)))
        return ms.value

    def size_bucket(self) -> str:
        """The autotuner's scene-size bucket: scene count and largest body and
        vertex counts, each rounded up to a power of two."""
        p2 = lambda v: 1 << max(0, int(v) - 1).bit_length()
        return (f"scenes{p2(len(self.scenes))}_bodies{p2(max(s.n_bodies for s in self.scenes))}"
                f"_verts{p2(max(s.n_vertices for s in self.scenes))}")

    def autotune(self, cache_path: str | None = None, steps: int = 2, candidates=AUTOTUNE_CTAS) -> dict:
        """Picks each queue-form kernel's persistent grid (CTAs per SM) by
        measurement and caches it in a JSON file keyed by device and size
        bucket.  A cached entry is applied without timing.  Otherwise a
        coordinate search: for each kernel in turn, each candidate is set,
        stepped once untimed (the graphs are rebuilt) and then `steps` times
        under CUDA events, and the fastest is kept.  The scenes advance while
        tuning; their results do not depend on the grids.  Returns
        {"key", "choice", "cached", "timings_ms"}."""
        import json
        sm, name = device_info()
        key = f"{name}|sm{sm}|{self.size_bucket()}"
        cache = {}
        if cache_path and os.path.exists(cache_path):
            with open(cache_path) as f:
                cache = json.load(f)
        if key in cache:
            choice = {k: int(v) for k, v in cache[key].items()}
            for kname, v in choice.items():
                self.set_queue_ctas(QUEUE_KERNELS[kname], v)
            return {"key": key, "choice": choice, "cached": True, "timings_ms": {}}
        choice = {k: 4 for k in QUEUE_KERNELS}
        timings = {}
        for kname, kid in QUEUE_KERNELS.items():
            best = None
            for cand in candidates:
                self.set_queue_ctas(kid, cand)
                self.step()
                ms = self.timed_steps(steps)
                timings[f"{kname}={cand}"] = ms
                if best is None or ms < best[1]:
                    best = (cand, ms)
            choice[kname] = best[0]
            self.set_queue_ctas(kid, best[0])
        if cache_path:
            cache[key] = choice
            tmp = cache_path + ".tmp"
            with open(tmp, "w") as f:
                json.dump(cache, f, indent=1, sort_keys=True)
            os.replace(tmp, cache_path)
        return {"key": key, "choice": choice, "cached": False, "timings_ms": timings}

    def state(self, i: int) -> dict:
        sb = abi.StateBuffers(self.scenes[i].n_bodies)
        v = sb.view()
        _check("nxd_batch_get_state", lib().nxd_batch_get_state(self.h, i, C.byref(v)))
        return sb.as_dict()

    def diagnostics(self, i: int) -> dict:
        d = abi.NxdDiagnostics()
        _check("nxd_batch_get_diagnostics", lib().nxd_batch_get_diagnostics(self.h, i, C.byref(d)))
        return d.as_dict()


def body_pairs_noalloc(position_ptr: int, orientation_ptr: int, local_box_ptr: int, n: int, r: float,
                       pairs_ptr: int, cap: int, stream_ptr: int = 0) -> int:
    """nxd_body_pairs_noalloc on caller-owned device buffers (raw pointers);
    returns the pair count."""
    cnt = C.c_int64(0)
    _check("nxd_body_pairs_noalloc", lib().nxd_body_pairs_noalloc(
        C.c_void_p(position_ptr), C.c_void_p(orientation_ptr), C.c_void_p(local_box_ptr), n, r,
        C.c_void_p(pairs_ptr), cap, C.byref(cnt), C.c_void_p(stream_ptr) if stream_ptr else None))
    return cnt.value


def fp64_peak(stream_ptr: int = 0):
    """nxd_fp64_peak: (TFLOP/s of FP64 FMA on the current device, ms)."""
    tf, ms = C.c_double(0), C.c_double(0)
    _check("nxd_fp64_peak", lib().nxd_fp64_peak(C.c_void_p(stream_ptr) if stream_ptr else None, C.byref(tf),
                                                C.byref(ms)))
    return tf.value, ms.value


class World:
    """World of the reference (Dynamics/World.h:11-17): a generated scene."""

    def __init__(self, scene):
        self.scene = scene


class IPCSolver:
    """IPCSolver facade (Dynamics/IPCSolver.h:21-91): settings are applied to
    the scene's nxd_settings before the device context is created on the
    first step(world, dt)."""

    def __init__(self):
        self._overrides = {}
        self.ctx = None

    def enableCCD(self, on: bool): self._overrides["enable_ccd"] = int(on)
    def setCCDSafetyFactor(self, f: float): self._overrides["ccd_safety_factor"] = float(f)
    def enableAdaptiveBarrier(self, on: bool): self._overrides["enable_adaptive_barrier"] = int(on)
    def enableFriction(self, on: bool): self._overrides["enable_friction"] = int(on)
    def setFrictionCoefficient(self, mu: float): self._overrides["friction_coeff"] = float(mu)
    def setContactDistanceThreshold(self, dhat: float): self._overrides["dhat"] = max(1e-9, float(dhat))
    def setContactStiffness(self, k: float):
        if k > 0.0:
            self._overrides["contact_stiffness"] = float(k)
    def setALMMaxIters(self, n: int): self._overrides["alm_max_iters"] = max(1, int(n))
    def setALMConstraintTolerance(self, t: float): self._overrides["alm_constraint_tol"] = max(1e-12, float(t))
    def setALMDualTolerance(self, t: float): self._overrides["alm_dual_tol"] = max(1e-12, float(t))
    def setALMContactTolerance(self, t: float): self._overrides["alm_contact_tol"] = max(1e-12, float(t))
    def setALMHardeningTrigger(self, t: float): self._overrides["alm_hardening_trigger"] = max(1.0, float(t))
    def setALMHardeningRatio(self, r: float): self._overrides["alm_hardening_ratio"] = max(1.0, float(r))

    def step(self, world: World, dt: float):
        if self.ctx is None:
            for k, v in self._overrides.items():
                setattr(world.scene.settings, k, v)
            self.ctx = Context(world.scene)
        self.ctx.step(dt)

    def diagnostics(self) -> dict:
        return self.ctx.diagnostics()

    def lastDualResidual(self): return self.diagnostics()["last_dual_residual"]
    def lastContactResidual(self): return self.diagnostics()["last_contact_residual"]
    def lastMaxConstraintViolation(self): return self.diagnostics()["last_max_constraint_violation"]
    def lastAngularVelocityError(self): return self.diagnostics()["last_angular_velocity_error"]
    def lastTorqueSaturationRatio(self): return self.diagnostics()["last_torque_saturation_ratio"]
