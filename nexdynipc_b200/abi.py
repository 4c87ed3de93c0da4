"""ctypes mirror of include/nxd.h (the C ABI of libnxd_b200.so).

Only plain C types cross the boundary: int32/int64/double pointers and the
structs below.  `SceneArrays.desc()` builds an `NxdSceneDesc` whose pointers
reference numpy arrays owned by the `SceneArrays` instance.
"""
from __future__ import annotations

import ctypes as C
import numpy as np

NXD_JOINT_HINGE = 0
NXD_JOINT_FIXED = 1
NXD_JOINT_SPHERICAL = 2
NXD_JOINT_ANGLE_LIMIT = 3
NXD_JOINT_PRISMATIC = 4
NXD_JOINT_CYLINDRICAL = 5
NXD_JOINT_DISTANCE_LIMIT = 6
NXD_JOINT_PARAMS = 16
NXD_DRIVE_PARAMS = 8
NXD_DRIVE_ANGULAR_VELOCITY = 0
NXD_DRIVE_LINEAR_VELOCITY = 1
NXD_DRIVE_POSITION = 2
NXD_DRIVE_FORCE = 3
NXD_DRIVE_DAMPED_SPRING = 4

NXD_FORM_INERTIA = 0
NXD_FORM_GRAVITY = 1
NXD_FORM_CONSTRAINT = 2
NXD_FORM_BARRIER = 3
NXD_FORM_FRICTION = 4
NXD_FORM_DRIVES = 5
NXD_FORM_TOTAL = 6
NXD_FORM_CONTACT = 7

STATUS_NAMES = {
    0: "NXD_OK", 1: "NXD_NOT_CONVERGED", 2: "NXD_LS_FAILED", 3: "NXD_FACTOR_FAILED",
    4: "NXD_CAPACITY", 5: "NXD_NAN", 6: "NXD_TIMEOUT", 7: "NXD_INVALID_ARGUMENT",
    8: "NXD_CUDA_ERROR", 9: "NXD_NO_DEVICE",
}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class NxdSettings(C.Structure):
    _fields_ = [
        ("dhat", C.c_double),
        ("contact_stiffness", C.c_double),
        ("enable_adaptive_barrier", C.c_int32),
        ("enable_ccd", C.c_int32),
        ("ccd_safety_factor", C.c_double),
        ("enable_friction", C.c_int32),
        ("alm_max_iters", C.c_int32),
        ("friction_coeff", C.c_double),
        ("alm_constraint_tol", C.c_double),
        ("alm_dual_tol", C.c_double),
        ("alm_contact_tol", C.c_double),
        ("alm_hardening_trigger", C.c_double),
        ("alm_hardening_ratio", C.c_double),
        ("newton_max_iters", C.c_int32),
        ("ls_max_iters", C.c_int32),
        ("newton_tol", C.c_double),
        ("ls_c1", C.c_double),
        ("ls_rho", C.c_double),
        ("integrator", C.c_int32),
        ("reserved0", C.c_int32),
        ("newmark_beta", C.c_double),
        ("newmark_gamma", C.c_double),
    ]

INTEGRATOR_IMPLICIT_EULER = 0
INTEGRATOR_IMPLICIT_NEWMARK = 1


def default_settings() -> NxdSettings:
    """IPCSolver / NewtonSolver / BacktrackingLineSearch defaults
    (Dynamics/IPCSolver.h:97-119, Math/NewtonSolver.h:58-64, Math/LineSearch.h:36-38)."""
    s = NxdSettings()
    s.dhat = 1e-3
    s.contact_stiffness = -1.0
    s.enable_adaptive_barrier = 1
    s.enable_ccd = 1
    s.ccd_safety_factor = 0.8
    s.enable_friction = 0
    s.alm_max_iters = 10
    s.friction_coeff = 0.0
    s.alm_constraint_tol = 1e-4
    s.alm_dual_tol = 1e-3
    s.alm_contact_tol = 1e-3
    s.alm_hardening_trigger = 2.0
    s.alm_hardening_ratio = 2.0
    s.newton_max_iters = 20
    s.ls_max_iters = 20
    s.newton_tol = 1e-6
    s.ls_c1 = 1e-4
    s.ls_rho = 0.5
    s.integrator = INTEGRATOR_IMPLICIT_EULER     # IPCSolver's own default (IPCSolver.cpp:264-266)
    s.newmark_beta = 0.25                        # ImplicitTimeIntegrator::create defaults
    s.newmark_gamma = 0.5
    return s


class NxdSceneDesc(C.Structure):
    _fields_ = [
        ("n_bodies", C.c_int32),
        ("body_ids", _ip),
        ("position", _dp),
        ("orientation", _dp),
        ("velocity", _dp),
        ("angular_velocity", _dp),
        ("linear_acceleration", _dp),
        ("angular_acceleration", _dp),
        ("mass", _dp),
        ("inertia_body", _dp),
        ("vertex_offset", _ip),
        ("vertices", _dp),
        ("face_offset", _ip),
        ("faces", _ip),
        ("n_joints", C.c_int32),
        ("joint_type", _ip),
        ("joint_body_a", _ip),
        ("joint_body_b", _ip),
        ("joint_params", _dp),
        ("joint_stiffness", _dp),
        ("n_drives", C.c_int32),
        ("drive_body_a", _ip),
        ("drive_body_b", _ip),
        ("drive_params", _dp),
        ("settings", NxdSettings),
        ("n_contact_pairs", C.c_int32),
        ("contact_pair_bodies", _ip),
        ("contact_pair_friction", _dp),
        ("drive_kind", _ip),
    ]


class NxdBsr(C.Structure):
    _fields_ = [
        ("n_rows", C.c_int32),
        ("nnzb", C.c_int64),
        ("row_ptr", _ip),
        ("col_idx", _ip),
        ("vals", _dp),
    ]


class NxdSolveStats(C.Structure):
    _fields_ = [
        ("components", C.c_int32),
        ("singletons", C.c_int32),
        ("largest_component", C.c_int32),
        ("factor_failed", C.c_int32),
    ]


class NxdPcgStats(C.Structure):
    _fields_ = [
        ("iterations", C.c_int32),
        ("status", C.c_int32),
        ("relative_residual", C.c_double),
        ("kernel_ms", C.c_double),
        ("grid", C.c_int32),
        ("threads", C.c_int32),
    ]


class NxdIpcParams(C.Structure):
    _fields_ = [
        ("dhat", C.c_double),
        ("kappa", C.c_double),
        ("eta", C.c_double),
        ("newton_tol", C.c_double),
        ("newton_max_iters", C.c_int32),
        ("ls_max_iters", C.c_int32),
        ("linear_solver", C.c_int32),
        ("pcg_max_iter", C.c_int32),
        ("pcg_tol", C.c_double),
        ("mu", C.c_double),
        ("friction_eps", C.c_double),
        ("friction_iters", C.c_int32),
        ("pad", C.c_int32),
    ]


class NxdIpcStats(C.Structure):
    _fields_ = [
        ("newton_iterations", C.c_int32),
        ("converged", C.c_int32),
        ("line_search_failed", C.c_int32),
        ("solve_failed", C.c_int32),
        ("last_alpha_max", C.c_double),
        ("energy", C.c_double),
        ("n_pairs", C.c_int64),
        ("n_active", C.c_int64),
        ("pcg_iterations", C.c_int64),
        ("n_friction", C.c_int64),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


IPC_SOLVER_DIRECT, IPC_SOLVER_PCG = 0, 1


def ipc_params(dhat=1e-3, kappa=1e8, eta=0.1, newton_tol=1e-6, newton_max_iters=50, ls_max_iters=30,
               linear_solver=IPC_SOLVER_DIRECT, pcg_max_iter=500, pcg_tol=1e-12, mu=0.0, friction_eps=1e-8,
               friction_iters=1) -> "NxdIpcParams":
    return NxdIpcParams(dhat, kappa, eta, newton_tol, newton_max_iters, ls_max_iters, linear_solver, pcg_max_iter,
                        pcg_tol, mu, friction_eps, friction_iters, 0)


class NxdIpcAdjointOut(C.Structure):
    _fields_ = [
        ("lam", _dp),
        ("phat_bar", _dp),
        ("thetahat_bar", _dp),
        ("phi_bar", _dp),
        ("mass_bar", _dp),
        ("inertia_bar", _dp),
        ("joint_mu_bar", _dp),
        ("n_active", C.POINTER(C.c_int32)),
        ("p0_bar", _dp),
        ("friction_mu_bar", _dp),
    ]


class NxdState(C.Structure):
    _fields_ = [
        ("position", _dp),
        ("orientation", _dp),
        ("velocity", _dp),
        ("angular_velocity", _dp),
        ("linear_acceleration", _dp),
        ("angular_acceleration", _dp),
    ]


class NxdContact(C.Structure):
    _fields_ = [
        ("point", C.c_double * 3),
        ("normal", C.c_double * 3),
        ("distance", C.c_double),
        ("body_a", C.c_int32),
        ("body_b", C.c_int32),
        ("primitive_type", C.c_int32),
        ("primitive_a", C.c_int32),
        ("primitive_b", C.c_int32),
        ("pad_", C.c_int32),
    ]


CONTACT_DTYPE = np.dtype([
    ("point", np.float64, 3), ("normal", np.float64, 3), ("distance", np.float64),
    ("body_a", np.int32), ("body_b", np.int32), ("primitive_type", np.int32),
    ("primitive_a", np.int32), ("primitive_b", np.int32), ("pad_", np.int32),
])
assert CONTACT_DTYPE.itemsize == C.sizeof(NxdContact) == 80


class NxdCandidates(C.Structure):
    _fields_ = [
        ("vv", _ip), ("vv_cap", C.c_int64), ("vv_count", C.c_int64),
        ("ev", _ip), ("ev_cap", C.c_int64), ("ev_count", C.c_int64),
        ("ee", _ip), ("ee_cap", C.c_int64), ("ee_count", C.c_int64),
        ("fv", _ip), ("fv_cap", C.c_int64), ("fv_count", C.c_int64),
    ]


class NxdDiagnostics(C.Structure):
    _fields_ = [
        ("kappa", C.c_double),
        ("dhat", C.c_double),
        ("actual_dt", C.c_double),
        ("last_dual_residual", C.c_double),
        ("last_contact_residual", C.c_double),
        ("last_max_constraint_violation", C.c_double),
        ("last_angular_velocity_error", C.c_double),
        ("last_torque_saturation_ratio", C.c_double),
        ("scene_min_distance", C.c_double),
        ("alm_iterations", C.c_int32),
        ("newton_iterations", C.c_int32),
        ("newton_converged", C.c_int32),
        ("n_body_pairs", C.c_int32),
        ("n_contacts", C.c_int32),
        ("n_contacts_raw", C.c_int32),
        ("status", C.c_int32),
        ("line_search_failures", C.c_int32),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_ip)


class StateBuffers:
    """Host arrays for one body state, plus the NxdState view over them."""

    def __init__(self, n: int):
        self.position = np.zeros((n, 3))
        self.orientation = np.zeros((n, 4))
        self.velocity = np.zeros((n, 3))
        self.angular_velocity = np.zeros((n, 3))
        self.linear_acceleration = np.zeros((n, 3))
        self.angular_acceleration = np.zeros((n, 3))

    def view(self) -> NxdState:
        return NxdState(dptr(self.position), dptr(self.orientation), dptr(self.velocity),
                        dptr(self.angular_velocity), dptr(self.linear_acceleration),
                        dptr(self.angular_acceleration))

    def as_dict(self) -> dict:
        return {k: getattr(self, k).copy() for k in
                ("position", "orientation", "velocity", "angular_velocity",
                 "linear_acceleration", "angular_acceleration")}

    def load(self, st: dict) -> "StateBuffers":
        for k, v in st.items():
            getattr(self, k)[...] = v
        return self
