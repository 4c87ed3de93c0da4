// adjoint.cuh — adjoint of the full-IPC time step (nxd_ipc_adjoint).
//
// The step solves G(x; z) = 0 for the iterate x = (p, theta) of every body
// (inertia, gravity, fixed joints, the primitive-pair barrier scaled by
// s = dt^2; rotational rows are the exact theta-gradient).  At the converged
// x*, the implicit function theorem turns output adjoints xbar = dL/dx* into
//   K^T lambda = xbar,  K = dG/dx (the exact Hessian of the step energy),
//   zbar = -(dG/dz)^T lambda
// for the step's inputs z: the predicted pose (p^ = p0 + dt v0, theta^ =
// dt w0), the step-start orientations (left rotations phi), the masses, the
// body inertias and the fixed joints' stiffnesses.
//
// Dense per world (6N <= 6 kAdjMaxBodies): one CTA assembles K^T and the
// orientation block K_phi in global memory, the pairs in candidate order
// (deterministic sums), one CTA solves by Gaussian elimination with partial
// pivoting, and the cross terms are column sums in fixed order.
#pragma once

#include "ipc.cuh"

namespace nx {

constexpr int kAdjMaxBodies = 128;
constexpr int kAdjThreads = 1024;

// J_r^-1(t) = I + [t]x / 2 + c [t]x^2, c = 1/phi^2 - (1 + cos phi) / (2 phi sin phi)
__device__ __forceinline__ void jr_inverse(V3 t, double* Ji) {
    const double phi = sqrt(dot(t, t));
    double c;
    if (phi < 1e-2) {
        const double p2 = phi * phi;
        c = 1.0 / 12.0 + p2 * (1.0 / 720.0) + (p2 * p2) * (1.0 / 30240.0);
    } else {
        double sn, cs;
        nxm::sincos(phi, &sn, &cs);
        c = 1.0 / (phi * phi) - (1.0 + cs) / (2.0 * phi * sn);
    }
    double S[9], S2[9];
    ipc::m3_skew(t, S);
    ipc::m3_mul(S, S, S2);
    for (int e = 0; e < 9; ++e) Ji[e] = (e % 4 == 0 ? 1.0 : 0.0) + 0.5 * S[e] + c * S2[e];
}

struct AdjIn {
    int N, J;
    const double* mass; const double* inertia;         // [N], [9N]
    const int* jtype; const int* ja; const double* jparams; const double* jmu;   // joints, stiffness used
    const double* quat0;                                // step-start orientations [4N]
    const double* xs;                                   // x* [6N]
    const double* xhat;                                 // predicted pose [6N]
    double s;                                           // barrier / gravity scale dt^2
};

// The frozen friction pairs' blocks (k_fric_pair_adjoint), when the step
// has friction: kp / kf like the barrier's, ks on the step-start positions
// and orientations, gm on mu.
struct AdjFric {
    int n;
    const int* body; const double* kp; const double* kf; const double* ks; const double* gm;
    double* Kps;    // [n6 x 3N] dG / d(step-start positions)
    double* gmu;    // [n6]      dG / d(mu)
};

// K^T (n x n) and K_phi (n x 3N), n = 6N; the pairs' blocks in pair order,
// then the friction pairs' in frozen order.
__global__ void __launch_bounds__(kAdjThreads) k_adj_assemble(AdjIn a, const int* pair_body, const int* pair_active,
                                                              const double* kp, const double* kf, int n_pairs, double* Kt,
                                                              double* Kphi, AdjFric fr) {
    const int n = 6 * a.N, m3 = 3 * a.N;
    for (long long e = threadIdx.x; e < (long long)n * n; e += blockDim.x) Kt[e] = 0.0;
    for (long long e = threadIdx.x; e < (long long)n * m3; e += blockDim.x) Kphi[e] = 0.0;
    if (fr.n) {
        for (long long e = threadIdx.x; e < (long long)n * m3; e += blockDim.x) fr.Kps[e] = 0.0;
        for (int e = threadIdx.x; e < n; e += blockDim.x) fr.gmu[e] = 0.0;
    }
    __syncthreads();
    // inertia: K[p][p] = m I, K[theta][theta] = I_body (K^T holds its transpose)
    for (int b = threadIdx.x; b < a.N; b += blockDim.x) {
        for (int i = 0; i < 3; ++i) {
            Kt[(size_t)(6 * b + i) * n + 6 * b + i] += a.mass[b];
            for (int j = 0; j < 3; ++j) Kt[(size_t)(6 * b + 3 + j) * n + 6 * b + 3 + i] += a.inertia[9 * b + 3 * i + j];
        }
    }
    __syncthreads();
    // fixed joints in joint order: mu I on the body's block, mu J_r^-1(tt) on
    // d G_theta / d phi (C_theta = theta - Log(q_t q0^-1))
    for (int j = 0; j < a.J; ++j) {
        if (a.jtype[j] != NXD_JOINT_FIXED) continue;
        const int A = a.ja[j];
        const double mu = a.jmu[j];
        if (threadIdx.x < 6) Kt[(size_t)(6 * A + threadIdx.x) * n + 6 * A + threadIdx.x] += mu;
        if (threadIdx.x == 32) {
            const Q dq = qmul(ldq(a.jparams + 16 * j + 3), qconj(ldq(a.quat0 + 4 * A)));
            double ang; V3 ax;
            q_to_angle_axis(dq, ang, ax);
            double Ji[9];
            jr_inverse(ax * ang, Ji);
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) Kphi[(size_t)(6 * A + 3 + r) * m3 + 3 * A + c] += mu * Ji[3 * r + c];
        }
        __syncthreads();
    }
    // pairs, in candidate order
    for (int p = 0; p < n_pairs; ++p) {
        if (!pair_active[p]) continue;
        const int bd[2] = {pair_body[2 * p], pair_body[2 * p + 1]};
        const int t = threadIdx.x;
        if (t < 144) {
            const int r = t / 12, c = t % 12;
            const int gr = 6 * bd[r / 6] + r % 6, gc = 6 * bd[c / 6] + c % 6;
            Kt[(size_t)gc * n + gr] += a.s * kp[144 * (size_t)p + t];
        } else if (t < 216) {
            const int u = t - 144, r = u / 6, c = u % 6;
            const int gr = 6 * bd[r / 6] + r % 6, gc = 3 * bd[c / 3] + c % 3;
            Kphi[(size_t)gr * m3 + gc] += a.s * kf[72 * (size_t)p + u];
        }
        __syncthreads();
    }
    for (int f = 0; f < fr.n; ++f) {
        const int bd[2] = {fr.body[2 * f], fr.body[2 * f + 1]};
        const int t = threadIdx.x;
        if (t < 144) {
            const int r = t / 12, c = t % 12;
            const int gr = 6 * bd[r / 6] + r % 6, gc = 6 * bd[c / 6] + c % 6;
            Kt[(size_t)gc * n + gr] += a.s * fr.kp[144 * (size_t)f + t];
        } else if (t < 216) {
            const int u = t - 144, r = u / 6, c = u % 6;
            const int gr = 6 * bd[r / 6] + r % 6, gc = 3 * bd[c / 3] + c % 3;
            Kphi[(size_t)gr * m3 + gc] += a.s * fr.kf[72 * (size_t)f + u];
        } else if (t < 228) {
            const int r = t - 216;
            fr.gmu[6 * bd[r / 6] + r % 6] += a.s * fr.gm[12 * (size_t)f + r];
        }
        __syncthreads();
        // ks columns (p_A, phi_A, p_B, phi_B): positions to Kps, orientations
        // to K_phi after kf's share of the same entries (no two threads on one)
        if (t < 144) {
            const int r = t / 12, c = t % 12;
            const int gr = 6 * bd[r / 6] + r % 6, cb = 3 * bd[c / 6] + c % 3;
            if (c % 6 < 3) fr.Kps[(size_t)gr * m3 + cb] += a.s * fr.ks[144 * (size_t)f + t];
            else Kphi[(size_t)gr * m3 + cb] += a.s * fr.ks[144 * (size_t)f + t];
        }
        __syncthreads();
    }
}

// A x = b by Gaussian elimination with partial pivoting (A n x n row-major,
// overwritten; ties of the pivot magnitude go to the lower row).  One CTA.
// *fail = 1 on a zero pivot.
__global__ void __launch_bounds__(kAdjThreads) k_adj_solve(double* A, double* b, int n, double* x, int* fail) {
    __shared__ double sv[32];
    __shared__ int si[32];
    __shared__ int piv;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5, nw = blockDim.x >> 5;
    if (t == 0) *fail = 0;
    for (int k = 0; k < n; ++k) {
        // pivot: max |A[i][k]|, i >= k
        double bv = -1.0;
        int bi = n;
        for (int i = k + t; i < n; i += blockDim.x) {
            const double v = fabs(A[(size_t)i * n + k]);
            if (v > bv || (v == bv && i < bi)) { bv = v; bi = i; }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
        }
        if (lane == 0) { sv[w] = bv; si[w] = bi; }
        __syncthreads();
        if (t == 0) {
            double v = sv[0];
            int i0 = si[0];
            for (int q = 1; q < nw; ++q)
                if (sv[q] > v || (sv[q] == v && si[q] < i0)) { v = sv[q]; i0 = si[q]; }
            piv = (v > 0.0 && i0 < n) ? i0 : -1;
            if (piv < 0) *fail = 1;
        }
        __syncthreads();
        const int pr = piv;
        if (pr < 0) return;
        if (pr != k) {
            for (int j = t; j < n; j += blockDim.x) {
                const double u = A[(size_t)k * n + j];
                A[(size_t)k * n + j] = A[(size_t)pr * n + j];
                A[(size_t)pr * n + j] = u;
            }
            if (t == 0) { const double u = b[k]; b[k] = b[pr]; b[pr] = u; }
        }
        __syncthreads();
        const double akk = A[(size_t)k * n + k];
        const int rows = n - k - 1;
        for (long long e = t; e < (long long)rows * (n - k); e += blockDim.x) {
            const int i = k + 1 + (int)(e / (n - k)), j = k + (int)(e % (n - k));
            const double l = A[(size_t)i * n + k] / akk;
            if (j == k) continue;
            A[(size_t)i * n + j] -= l * A[(size_t)k * n + j];
        }
        __syncthreads();
        for (int i = k + 1 + t; i < n; i += blockDim.x) {
            const double l = A[(size_t)i * n + k] / akk;
            b[i] -= l * b[k];
            A[(size_t)i * n + k] = 0.0;
        }
        __syncthreads();
    }
    // back substitution, row by row (the row's dot product over the CTA)
    for (int i = n - 1; i >= 0; --i) {
        double acc = 0.0;
        for (int j = i + 1 + t; j < n; j += blockDim.x) acc += A[(size_t)i * n + j] * x[j];
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) sv[w] = acc;
        __syncthreads();
        if (t == 0) {
            double s = 0.0;
            for (int q = 0; q < nw; ++q) s += sv[q];
            x[i] = (b[i] - s) / A[(size_t)i * n + i];
        }
        __syncthreads();
    }
}

struct AdjOut {
    double* phat_bar;       // [3N]  m lambda_p
    double* thetahat_bar;   // [3N]  I^T lambda_theta
    double* phi_bar;        // [3N]  -(K_phi^T lambda)
    double* mass_bar;       // [N]
    double* inertia_bar;    // [9N]  -lambda_theta (theta - theta^)^T
    double* joint_mu_bar;   // [J]   -lambda_A . C
    double* p0_bar;         // [3N]  -(K_ps^T lambda) (friction)
    double* friction_mu_bar;// [1]   -lambda . dG/dmu (friction)
};

__global__ void k_adj_cross(AdjIn a, const double* lam, const double* Kphi, AdjOut o, AdjFric fr) {
    const int n = 6 * a.N, m3 = 3 * a.N;
    const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
    for (int c = gt; c < m3; c += gs) {
        double acc = 0.0;
        for (int r = 0; r < n; ++r) acc += Kphi[(size_t)r * m3 + c] * lam[r];
        o.phi_bar[c] = -acc;
        double ap = 0.0;
        if (fr.n)
            for (int r = 0; r < n; ++r) ap += fr.Kps[(size_t)r * m3 + c] * lam[r];
        o.p0_bar[c] = -ap;
    }
    if (gt == 0) {
        double acc = 0.0;
        if (fr.n)
            for (int r = 0; r < n; ++r) acc += fr.gmu[r] * lam[r];
        *o.friction_mu_bar = -acc;
    }
    for (int b = gt; b < a.N; b += gs) {
        const double* L = lam + 6 * b;
        const double* x = a.xs + 6 * b;
        const double* xh = a.xhat + 6 * b;
        const double m = a.mass[b];
        const double g[3] = {0.0, -9.81, 0.0};
        double mb = 0.0;
        for (int i = 0; i < 3; ++i) {
            o.phat_bar[3 * b + i] = m * L[i];
            double th = 0.0;
            for (int j = 0; j < 3; ++j) th += a.inertia[9 * b + 3 * j + i] * L[3 + j];
            o.thetahat_bar[3 * b + i] = th;
            mb += L[i] * ((x[i] - xh[i]) - a.s * g[i]);
            for (int j = 0; j < 3; ++j) o.inertia_bar[9 * b + 3 * i + j] = -(L[3 + i] * (x[3 + j] - xh[3 + j]));
        }
        o.mass_bar[b] = -mb;
    }
    for (int j = gt; j < a.J; j += gs) {
        if (a.jtype[j] != NXD_JOINT_FIXED) { o.joint_mu_bar[j] = 0.0; continue; }
        const int A = a.ja[j];
        const double* P = a.jparams + 16 * j;
        const Q dq = qmul(ldq(P + 3), qconj(ldq(a.quat0 + 4 * A)));
        double ang; V3 ax;
        q_to_angle_axis(dq, ang, ax);
        const V3 tt = ax * ang;
        const double* x = a.xs + 6 * A;
        const double C[6] = {x[0] - P[0], x[1] - P[1], x[2] - P[2], x[3] - tt.x, x[4] - tt.y, x[5] - tt.z};
        double acc = 0.0;
        for (int k = 0; k < 6; ++k) acc += lam[6 * A + k] * C[k];
        o.joint_mu_bar[j] = -acc;
    }
}

}  // namespace nx
