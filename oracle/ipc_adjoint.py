"""CPU restatement of the full-IPC time step's adjoint (test infrastructure:
the checker of the device adjoint, nxd_ipc_adjoint; only tests/ and bench.py's
CPU leg use it).

The step (nxo_ipc_step / nxd_ipc_step, implicit Euler) solves G(x; z) = 0 for
the iterate x = (p, theta) of every body, with
  G = inertia [m (p - p^), I (theta - theta^)]  (p^ = p0 + dt v0, theta^ = dt w0)
    + gravity s [-m g, 0]
    + fixed joints  lambda + mu C  (C = [p - p_t, theta - log(q_t q0^-1)])
    + s * barrier (per pair: point forces g_k, body torques a_k x g_k),
s = dt^2, world points w_k = p + Exp(theta) R(q0) r_k, arms a_k = w_k - p.
The implicit function theorem gives, for output adjoints xbar of x*,
  K^T lambda = xbar,   K = dG/dx at x*,   zbar = -(dG/dz)^T lambda.
G's rotational rows are the exact theta-gradient, J_r(theta) times the
lever-arm torque (ipc_pair.h chain12_exact), so K is the exact, symmetric
Hessian of the step's energy: the pair Hessian unprojected (oracle
raw_hessian) chained by d(Exp(theta) v)/dtheta = -[Exp(theta) v]x J_l(theta),
plus the derivatives of the arms and of J_r(theta).  Orientation inputs are
perturbed on the left, q0 -> Exp(phi) q0, and their adjoints are tangent
3-vectors.

No reference code is restated here: the reference has no adjoint (its
differentiable-physics plan, documents/2026.02.21, is unimplemented).
"""
from __future__ import annotations

import numpy as np

from nexdynipc_b200 import abi
from . import refcpu

GRAVITY = np.array([0.0, -9.81, 0.0])


def skew(v):
    return np.array([[0.0, -v[2], v[1]], [v[2], 0.0, -v[0]], [-v[1], v[0], 0.0]])


def quat_mat(q):
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                     [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                     [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


def exp_mat(th):
    a = np.linalg.norm(th)
    if a < 1e-12:
        return np.eye(3) + skew(th)
    K = skew(th / a)
    return np.eye(3) + np.sin(a) * K + (1 - np.cos(a)) * K @ K


def jr_coeffs(a):
    """c1, c2 of J_r and d1 = c1'(a)/a, d2 = c2'(a)/a."""
    if a < 1e-2:
        a2 = a * a
        c1 = 0.5 - a2 / 24.0 + a2 * a2 / 720.0
        c2 = 1.0 / 6.0 - a2 / 120.0 + a2 * a2 / 5040.0
        d1 = -2.0 / 24.0 + 4.0 * a2 / 720.0 - 6.0 * a2 * a2 / 40320.0
        d2 = -2.0 / 120.0 + 4.0 * a2 / 5040.0 - 6.0 * a2 * a2 / 362880.0
        return c1, c2, d1, d2
    s, c = np.sin(a), np.cos(a)
    c1, c2 = (1 - c) / a ** 2, (a - s) / a ** 3
    d1 = s / a ** 3 - 2 * (1 - c) / a ** 4
    d2 = (1 - c) / a ** 4 - 3 * (a - s) / a ** 5
    return c1, c2, d1, d2


def right_jacobian(th):
    """J_r = J_l^T: the exact theta-gradient of an energy of world points is
    J_r(theta) times the lever-arm torque."""
    c1, c2, _, _ = jr_coeffs(np.linalg.norm(th))
    S = skew(th)
    return np.eye(3) - c1 * S + c2 * S @ S


def left_jacobian(th):
    """J_l: Exp(th + d) = Exp(J_l(th) d) Exp(th) to first order."""
    return right_jacobian(th).T


def jr_torque_derivative(th, tau):
    """M = d(J_r(theta) tau)/dtheta at fixed tau."""
    c1, c2, d1, d2 = jr_coeffs(np.linalg.norm(th))
    tt = np.cross(th, tau)
    ttt = np.cross(th, tt)
    return (-np.outer(tt, d1 * th) + c1 * skew(tau) + np.outer(ttt, d2 * th)
            + c2 * (np.dot(th, tau) * np.eye(3) + np.outer(th, tau) - 2 * np.outer(tau, th)))


def right_jacobian_inv(th):
    """J_r^-1: Log(Exp(th) Exp(d)) = th + J_r^-1(th) d to first order."""
    a = np.linalg.norm(th)
    S = skew(th)
    if a < 1e-4:
        c = 1.0 / 12.0 + a * a / 720.0
    else:
        c = 1.0 / (a * a) - (1 + np.cos(a)) / (2 * a * np.sin(a))
    return np.eye(3) + 0.5 * S + c * S @ S


def quat_mul(a, b):
    aw, ax, ay, az = a
    bw, bx, by, bz = b
    return np.array([aw * bw - ax * bx - ay * by - az * bz, aw * bx + ax * bw + ay * bz - az * by,
                     aw * by + ay * bw + az * bx - ax * bz, aw * bz + az * bw + ax * by - ay * bx])


def quat_log(q):
    """Angle-axis vector of q (FixedJoint's q_to_angle_axis: shortest angle)."""
    v = np.asarray(q[1:], dtype=np.float64)
    n = np.linalg.norm(v)
    if n == 0.0:
        return np.zeros(3)
    ang = 2 * np.arctan2(n, abs(q[0]))
    if q[0] < 0:
        n = -n
    return v / n * ang


def quat_tangent_adjoint(q, qbar):
    """psibar = (d(Exp(psi) q)/dpsi at 0)^T qbar for a 4-vector gradient qbar."""
    w, v = q[0], np.asarray(q[1:])
    return 0.5 * (w * qbar[1:] + np.cross(v, qbar[1:]) - qbar[0] * v)


def closest_weights(kind: int, typ: int, X):
    """The DistForm weights w (r = sum_k w_k X_k) of a pair of distance type
    `typ` (ipc_pair.h's codes) as a differentiable torch function of its
    four points X (4, 3)."""
    import torch
    w = [X.new_zeros(()) for _ in range(4)]
    one = X.new_ones(())
    if kind == 0:
        if typ == 6:
            e1, e2, q = X[2] - X[1], X[3] - X[1], X[0] - X[1]
            a, b, c, d, e = e1 @ e1, e1 @ e2, e2 @ e2, e1 @ q, e2 @ q
            det = a * c - b * b
            b1, b2 = (c * d - b * e) / det, (a * e - b * d) / det
            w = [one, -(1.0 - b1 - b2), -b1, -b2]
        elif typ in (3, 4, 5):
            i, j = [(1, 2), (2, 3), (3, 1)][typ - 3]
            ed = X[j] - X[i]
            t = (X[0] - X[i]) @ ed / (ed @ ed)
            w[0], w[i], w[j] = one, -(1.0 - t), -t
        else:
            w[0], w[typ + 1] = one, -one
    else:
        d1, d2, r = X[1] - X[0], X[3] - X[2], X[0] - X[2]
        if typ == 8:
            A, B, E, C, F = d1 @ d1, d1 @ d2, d2 @ d2, d1 @ r, d2 @ r
            sp = (B * F - C * E) / (A * E - B * B)
            tp = (B * sp + F) / E
            w = [1.0 - sp, sp, -(1.0 - tp), -tp]
        elif typ in (4, 5):
            pb = typ - 2
            sp = (X[pb] - X[0]) @ d1 / (d1 @ d1)
            w[0], w[1], w[pb] = 1.0 - sp, sp, -one
        elif typ in (6, 7):
            pa = typ - 6
            tp = (X[pa] - X[2]) @ d2 / (d2 @ d2)
            w[pa], w[2], w[3] = one, -(1.0 - tp), -tp
        else:
            w[typ // 2], w[2 + typ % 2] = one, -one
    return torch.stack([torch.as_tensor(v, dtype=X.dtype) for v in w])


def friction_force(kind, typ, X, Xs, dhat, kappa, mu, eps):
    """Point forces (12) of the lagged friction of one pair (ipc_pair.h's
    friction_pair without the |u| < 1e-12 branch) as a torch function of the
    points X at the iterate and Xs at the lag state (also the step start)."""
    import torch
    w = closest_weights(kind, typ, Xs)
    r = (w[:, None] * Xs).sum(0)
    s2 = r @ r
    d = torch.sqrt(s2)
    n = r / d
    sh = dhat * dhat
    b1 = -kappa * (2.0 * (s2 - sh) * torch.log(s2 / sh) + (s2 - sh) ** 2 / s2)
    lam = -2.0 * d * b1
    dsum = (w[:, None] * (X - Xs)).sum(0)
    u = dsum - (dsum @ n) * n
    s = torch.sqrt(u @ u + eps * eps)
    h = mu * lam * u / s
    return (w[:, None] * h[None, :]).reshape(12)


class StepAdjoint:
    """Adjoint of one full-IPC step of `scene` (barrier dhat, kappa): fixed
    joints and bodies only (no other joints, no control forms).  With
    friction mu > 0 (one lagging pass: the pairs frozen at the step start,
    eps), the frozen quantities' dependence on the start state is included
    (their derivatives by torch autograd of friction_force)."""

    def __init__(self, scene, dhat: float, kappa: float, mu: float = 0.0, eps: float = 1e-5):
        jt = np.asarray(scene.joint_type)
        if np.any(jt != abi.NXD_JOINT_FIXED) or len(scene.drive_body_b):
            raise ValueError("the step adjoint supports fixed joints and no control forms")
        self.sc = scene
        self.dhat, self.kappa = dhat, kappa
        self.mu, self.eps = mu, eps
        self.ow = refcpu.OracleWorld(scene)
        self.vbody, self.fbody, self.fvert, self.ebody, self.evert = self.ow.prim_topology()

    def pairs(self, xs):
        """Active pairs at x*: (kind, vertex ids [4], body per point, [bA, bB])."""
        pt, ee = self.ow.ipc_candidates(xs, None, self.dhat)
        out = []
        for v, f in pt:
            out.append((0, [v, *self.fvert[f]], [0, 1, 1, 1], (self.vbody[v], self.fbody[f])))
        for e0, e1 in ee:
            out.append((1, [*self.evert[e0], *self.evert[e1]], [0, 0, 1, 1], (self.ebody[e0], self.ebody[e1])))
        return out

    def __call__(self, state0: dict, xs, xbar, dt: float, mass=None, mu=None):
        """One step's adjoint at its converged iterate xs (6N) from the
        start state state0, for xbar = dL/dx*.  mass / mu default to the
        scene's.  Returns a dict: lam (6N), phat_bar (N,3) = m lam_p,
        thetahat_bar (N,3) = I^T lam_theta, phi_bar (N,3), mass_bar (N),
        inertia_bar (N,3,3), joint_mu_bar (J)."""
        sc = self.sc
        N = sc.n_bodies
        s = dt * dt
        m = np.asarray(sc.mass if mass is None else mass, dtype=np.float64)
        mus = np.asarray(sc.joint_stiffness if mu is None else mu, dtype=np.float64)
        Ib = np.asarray(sc.inertia, dtype=np.float64).reshape(N, 3, 3)
        self.ow.set_state(state0)
        q0 = np.asarray(state0["orientation"])
        xs = np.asarray(xs, dtype=np.float64)
        th = xs.reshape(N, 6)[:, 3:]
        Rth = [exp_mat(t) for t in th]
        JL = [left_jacobian(t) for t in th]
        wv, pos = self.ow.world_vertices_at(xs)
        K = np.zeros((6 * N, 6 * N))
        Kphi = np.zeros((6 * N, 3 * N))
        for b in range(N):
            K[6 * b:6 * b + 3, 6 * b:6 * b + 3] += m[b] * np.eye(3)
            K[6 * b + 3:6 * b + 6, 6 * b + 3:6 * b + 6] += Ib[b]
        jparams = np.asarray(sc.joint_params).reshape(-1, 16)
        Cj = []
        for j in range(len(sc.joint_type)):
            A = int(sc.joint_body_a[j])
            K[6 * A:6 * A + 6, 6 * A:6 * A + 6] += mus[j] * np.eye(6)
            dq = quat_mul(jparams[j, 3:7], q0[A] * np.array([1.0, -1.0, -1.0, -1.0]))
            tt = quat_log(dq)
            Kphi[6 * A + 3:6 * A + 6, 3 * A:3 * A + 3] += mus[j] * right_jacobian_inv(tt)
            Cj.append(np.concatenate([xs[6 * A:6 * A + 3] - jparams[j, :3], xs[6 * A + 3:6 * A + 6] - tt]))
        def chain_pair(g, H, X, side, bodies):
            """The pair's exact share of dG/dx (12 x 12) and of dG/dphi
            (12 x 6) for point forces g and their point Jacobian H, and the
            point-velocity map E."""
            E = np.zeros((12, 12))
            F = np.zeros((12, 6))
            arms = [X[k] - pos[bodies[side[k]]] for k in range(4)]
            for k in range(4):
                sg, a, b = side[k], arms[k], bodies[side[k]]
                E[3 * k:3 * k + 3, 6 * sg:6 * sg + 3] = np.eye(3)
                E[3 * k:3 * k + 3, 6 * sg + 3:6 * sg + 6] = -skew(a) @ JL[b]
                F[3 * k:3 * k + 3, 3 * sg:3 * sg + 3] = -skew(a) @ Rth[b]
            Kp = E.T @ H @ E
            Kf = E.T @ H @ F
            # derivative of the arms and of J_r(theta) in G_theta = J_r(theta) sum_k a_k x g_k
            for sg in range(2):
                b = bodies[sg]
                Jr = JL[b].T
                GA = np.zeros((3, 3))
                tau = np.zeros(3)
                for k in range(4):
                    if side[k] != sg:
                        continue
                    gk = g[3 * k:3 * k + 3]
                    GA += skew(gk) @ skew(arms[k])
                    tau += np.cross(arms[k], gk)
                Kp[6 * sg + 3:6 * sg + 6, 6 * sg + 3:6 * sg + 6] += Jr @ GA @ JL[b] + jr_torque_derivative(th[b], tau)
                Kf[6 * sg + 3:6 * sg + 6, 3 * sg:3 * sg + 3] += Jr @ GA @ Rth[b]
            return Kp, Kf, E

        def scatter(Kp, Kf, bodies):
            for si in range(2):
                for sj in range(2):
                    bi, bj = bodies[si], bodies[sj]
                    K[6 * bi:6 * bi + 6, 6 * bj:6 * bj + 6] += s * Kp[6 * si:6 * si + 6, 6 * sj:6 * sj + 6]
                    Kphi[6 * bi:6 * bi + 6, 3 * bj:3 * bj + 3] += s * Kf[6 * si:6 * si + 6, 3 * sj:3 * sj + 3]

        for kind, vid, side, bodies in self.pairs(xs):
            X = wv[vid]
            ev = refcpu.ipc_pair(kind, X, self.dhat, self.kappa)
            if not (ev["d2"] < self.dhat ** 2):
                continue
            Kp, Kf, _ = chain_pair(ev["g"], ev["H_raw"], X, side, bodies)
            scatter(Kp, Kf, bodies)
        # lagged friction (one pass): the pairs active at the step start, their
        # point forces and point Jacobians (with respect to the iterate's
        # points and to the step-start points, which are the lag state and the
        # displacements' origin) by autograd; the step-start points move with
        # the start positions and, on the left, with the orientations
        Kps = np.zeros((6 * N, 3 * N))     # dG / d(step-start positions)
        g_mu = np.zeros(6 * N)             # dG / d(mu)
        if self.mu > 0.0:
            import torch
            x_start = np.zeros(6 * N)
            x_start.reshape(N, 6)[:, :3] = np.asarray(state0["position"])
            ws, pos_s = self.ow.world_vertices_at(x_start)
            args = (self.dhat, self.kappa, self.mu, self.eps)
            for kind, vid, side, bodies in self.pairs(x_start):
                Xs = ws[vid]
                ev = refcpu.ipc_pair(kind, Xs, self.dhat, self.kappa)
                if not (ev["d2"] < self.dhat ** 2):
                    continue
                typ = int(ev["type"])
                Xt = torch.tensor(wv[vid])
                Xst = torch.tensor(Xs)
                fn = lambda a, b_: friction_force(kind, typ, a, b_, *args)
                g = fn(Xt, Xst).detach().numpy()
                H, Hs = (j.reshape(12, 12).detach().numpy()
                         for j in torch.autograd.functional.jacobian(fn, (Xt, Xst)))
                Kp, Kf, E = chain_pair(g, H, wv[vid], side, bodies)
                scatter(Kp, Kf, bodies)
                S = np.zeros((12, 12))     # step-start points from (p_A, phi_A, p_B, phi_B)
                for k in range(4):
                    sg = side[k]
                    a_s = Xs[k] - pos_s[bodies[sg]]
                    S[3 * k:3 * k + 3, 6 * sg:6 * sg + 3] = np.eye(3)
                    S[3 * k:3 * k + 3, 6 * sg + 3:6 * sg + 6] = -skew(a_s)
                Ks = E.T @ Hs @ S
                Gm = E.T @ g / self.mu
                for si in range(2):
                    bi = bodies[si]
                    g_mu[6 * bi:6 * bi + 6] += s * Gm[6 * si:6 * si + 6]
                    for sj in range(2):
                        bj = bodies[sj]
                        Kps[6 * bi:6 * bi + 6, 3 * bj:3 * bj + 3] += s * Ks[6 * si:6 * si + 6, 6 * sj:6 * sj + 3]
                        Kphi[6 * bi:6 * bi + 6, 3 * bj:3 * bj + 3] += s * Ks[6 * si:6 * si + 6, 6 * sj + 3:6 * sj + 6]
        lam = np.linalg.solve(K.T, np.asarray(xbar, dtype=np.float64))
        L = lam.reshape(N, 6)
        p0, v0, w0 = (np.asarray(state0[k]) for k in ("position", "velocity", "angular_velocity"))
        phat = p0 + dt * v0
        that = dt * w0
        xp, xt = xs.reshape(N, 6)[:, :3], th
        out = {"lam": lam, "K": K, "Kphi": Kphi,
               "phat_bar": m[:, None] * L[:, :3],
               "thetahat_bar": np.einsum("bji,bj->bi", Ib, L[:, 3:]),
               "phi_bar": -(Kphi.T @ lam).reshape(N, 3),
               "mass_bar": -np.einsum("bi,bi->b", L[:, :3], (xp - phat) - s * GRAVITY[None, :] * 1.0),
               "inertia_bar": -np.einsum("bi,bj->bij", L[:, 3:], xt - that),
               "joint_mu_bar": np.array([-L[int(sc.joint_body_a[j])] @ Cj[j] for j in range(len(sc.joint_type))]),
               "p0_bar": -(Kps.T @ lam).reshape(N, 3), "Kps": Kps, "g_mu": g_mu,
               "friction_mu_bar": float(-(lam @ g_mu))}
        return out
