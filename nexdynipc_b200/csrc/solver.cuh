// solver.cuh — the Newton solve of one ALM iteration as one CTA.
//
// Mirrors NewtonSolver::minimize (src/Math/NewtonSolver.cpp:10-95) over the
// SimulationProblem energy (src/Dynamics/IPCSolver.cpp:137-262):
//   E(x) = Inertia + h^2 Gravity + Constraint + sum_forms h^2 Form
// with BacktrackingLineSearch (src/Math/LineSearch.cpp:6-58), followed by the
// ALM bookkeeping of IPCSolver::step (IPCSolver.cpp:1084-1110).
//
// Arithmetic order (so the CPU oracle and this kernel round identically):
//  * gradient and Hessian entries accumulate their contributions in item
//    order (joints, drives, barrier contacts, friction contacts), gathered per
//    body from incidence lists sorted by item index;
//  * reductions over bodies / joints / contacts / DOFs use one fixed pairwise
//    tree (pad to a power of two, v[i] += v[i+h], h = P/2 .. 1);
//  * the linear solve is an LDL^T per connected block component, members
//    ordered by (distinct coupled neighbours, body index), right-looking
//    updates A_ic -= (L_ij L_cj) d_j in ascending j, forward substitution in
//    ascending and backward substitution in descending column order.
#pragma once

#include "nx_math.cuh"
#include "geometry.cuh"

namespace nx {

constexpr int kSolverThreads = 1024;
constexpr int kMaxComponentBodies = 256;

struct Drv {   // velocity drive parameters (VelocityDriveForm)
    double ax, ay, az, kv, vt, maxT, delay, tau;
};

struct Solver {
    int N, J, D, Cmax;
    // bodies
    const double* mass; const double* inertia;
    const double* pos0; const double* quat0;      // step-start pose (joint / friction references)
    double* x; const double* xhat;                // [6N]
    // joints
    const int* jtype; const int* ja; const int* jb; const double* jparams;
    double* jmu; double* jlam;
    const int* jinc_off; const int* jinc;         // body -> (joint*2+side), joint order
    // drives
    const int* da; const int* db; const Drv* dprm;
    double* dprevA; double* dprevB; int* dhas_prev; const double* dfilt;
    const int* dinc_off; const int* dinc;         // body -> (drive*2+side)
    // contacts
    const ContactRec* contacts; const int* ncontacts_ptr;
    const double* nforce; const int* nnf_ptr;
    int* cinc_off; int* cinc; int* cinc_cnt;      // built per ALM iteration
    // scalars
    const double* dt_ptr; const double* bdhat_ptr; const double* bkappa_ptr;
    const int* barrier_in_forms_ptr; const int* friction_form_ptr;
    double friction_mu, friction_eps;
    int newton_max_iters, ls_max_iters;
    double newton_tol, ls_c1, ls_rho;
    double alm_constraint_tol, alm_hardening_trigger, alm_hardening_ratio;
    // scratch
    double* g; double* cg; double* dx; double* xt; double* red;   // red: >= pow2(max(N,J,C, 6N)) doubles
    double* qj; double* qg;                                        // [N*4] poses at the evaluation point
    double* jC; double* jF; double* jJ; double* jE; int* jact;     // joints
    double* bD; double* bGP; double* bHP; double* bE;               // barrier per contact
    double* fFG; double* fHF; double* fJA; double* fJB; double* fE; // friction per contact
    double* dE; double* dG; double* dH;                            // drives
    double* Hd;                                                    // [N*36] diagonal blocks
    int* parent; int* comp; int* comp_size; int* comp_off; int* members; int* local;
    int* items; int* item_comp_off; int* item_list; int* n_items_ptr;
    int* deg;
    double* pool; long long pool_cap; long long* pool_off;
    unsigned char* nzb; long long nzb_cap; long long* nzb_off;
    int* cand; int cand_stride;
    double* dvec;                                                  // [12N] per-component rhs and pivots
    // outputs / state
    int* alm_done; int* status; int* newton_iters; int* converged; int* ls_fail;
    double* alm_mcv; double* alm_dual;
};

// ---------------------------------------------------------------------------
// Block-level helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ int pow2_ceil(int n) { int p = 1; while (p < n) p <<= 1; return p; }

// Fixed-tree sum of buf[0..n) (buf capacity >= pow2_ceil(n)); all threads call.
__device__ double block_tree_sum(double* buf, int n) {
    const int P = pow2_ceil(max(n, 1));
    for (int i = n + threadIdx.x; i < P; i += blockDim.x) buf[i] = 0.0;
    __syncthreads();
    for (int h = P / 2; h >= 1; h >>= 1) {
        for (int i = threadIdx.x; i < h; i += blockDim.x) buf[i] = buf[i] + buf[i + h];
        __syncthreads();
    }
    const double r = buf[0];
    __syncthreads();
    return r;
}

__device__ double block_max(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v = dmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        double w = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) w = dmax(w, __shfl_xor_sync(0xffffffffu, w, o));
        if (threadIdx.x == 0) sh[0] = w;
    }
    __syncthreads();
    const double r = sh[0];
    __syncthreads();
    return r;
}

// ---------------------------------------------------------------------------
// Per-item evaluation
// ---------------------------------------------------------------------------
__device__ __forceinline__ V3 xs3(const double* x, int i) { return ld3(x + i); }

// Joint C (and J, f if full).  J is dim x 12: columns 0-5 body A, 6-11 body B.
__device__ void joint_eval(const Solver& S, int j, const double* x, bool full) {
    const int t = S.jtype[j];
    const int A = S.ja[j], B = S.jb[j];
    const double* P = S.jparams + 16 * j;
    double C[6] = {0, 0, 0, 0, 0, 0};
    double Jm[6][12];
    if (full) for (int r = 0; r < 6; ++r) for (int c = 0; c < 12; ++c) Jm[r][c] = 0.0;
    int dim = 6;
    if (t == NXD_JOINT_HINGE || t == NXD_JOINT_SPHERICAL) {
        dim = t == NXD_JOINT_HINGE ? 6 : 3;
        const V3 pA = xs3(x, 6 * A), pB = xs3(x, 6 * B);
        const Q qA = ldq(S.qj + 4 * A), qB = ldq(S.qj + 4 * B);
        const V3 rA = qrot(qA, ld3(P)), rB = qrot(qB, ld3(P + 3));
        const V3 v = (pA + rA) - (pB + rB);
        C[0] = v.x; C[1] = v.y; C[2] = v.z;
        if (full) {
            // PointPrimitive::addJacobianRows (JointPrimitives.h:58-90)
            const M3 dA = cross_mat(rA), dB = cross_mat(rB);
            for (int i = 0; i < 3; ++i) {
                Jm[i][i] = 1.0; Jm[i][6 + i] = -1.0;
                for (int k = 0; k < 3; ++k) { Jm[i][3 + k] = -at(dA, i, k); Jm[i][9 + k] = at(dB, i, k); }
            }
        }
        if (t == NXD_JOINT_HINGE) {
            const V3 nA = qrot(qA, ld3(P + 6)), nB = qrot(qB, ld3(P + 9));
            const V3 c = cross(nA, nB);
            C[3] = c.x; C[4] = c.y; C[5] = c.z;
            if (full) {
                // AxisCrossPrimitive::addJacobianRows (JointPrimitives.h:212-240)
                const M3 mA = mat_mul(cross_mat(nB), cross_mat(nA));
                M3 na = cross_mat(nA);
                for (int k = 0; k < 9; ++k) na.m[k] = -na.m[k];
                const M3 mB = mat_mul(na, cross_mat(nB));
                for (int i = 0; i < 3; ++i)
                    for (int k = 0; k < 3; ++k) { Jm[3 + i][3 + k] = at(mA, i, k); Jm[3 + i][9 + k] = at(mB, i, k); }
            }
        }
    } else if (t == NXD_JOINT_FIXED) {
        // FixedJoint::computeC / computeJ (FixedJoint.cpp:23-56)
        const V3 p = xs3(x, 6 * A);
        const V3 d = p - ld3(P);
        C[0] = d.x; C[1] = d.y; C[2] = d.z;
        const Q dq = qmul(ldq(P + 3), qconj(ldq(S.quat0 + 4 * A)));
        double ang; V3 ax;
        q_to_angle_axis(dq, ang, ax);
        const V3 tt = ax * ang;
        const V3 th = xs3(x, 6 * A + 3);
        C[3] = th.x - tt.x; C[4] = th.y - tt.y; C[5] = th.z - tt.z;
        if (full) for (int i = 0; i < 6; ++i) Jm[i][i] = 1.0;
    } else {
        // AngleLimitJoint (AngleLimitJoint.cpp:45-96)
        dim = 2;
        const Q qA = ldq(S.qj + 4 * A), qB = ldq(S.qj + 4 * B);
        const Q qr = qmul(qconj(qA), qB);
        double ang; V3 ax;
        q_to_angle_axis(qr, ang, ax);
        const V3 axis = ld3(P);
        const double a = ang * dot(ax, axis);
        C[0] = P[3] - a;
        C[1] = a - P[4];
        if (full) {
            for (int k = 0; k < 3; ++k) {
                Jm[0][3 + k] = get(axis, k); Jm[1][3 + k] = -get(axis, k);
                Jm[0][9 + k] = -get(axis, k); Jm[1][9 + k] = get(axis, k);
            }
        }
    }
    const double mu = S.jmu[j];
    const double* lam = S.jlam + 6 * j;
    double* Cj = S.jC + 6 * j;
    for (int i = 0; i < 6; ++i) Cj[i] = C[i];
    // energy (Joint::value, Joint.cpp:5-18; AngleLimitJoint::value, AngleLimitJoint.cpp:98-109)
    if (t == NXD_JOINT_ANGLE_LIMIT) {
        double e = 0.0;
        for (int i = 0; i < 2; ++i) { const double gp = dmax(C[i], 0.0); e += lam[i] * gp + 0.5 * mu * gp * gp; }
        S.jE[j] = e;
    } else {
        double t1 = 0.0, sq = 0.0;
        for (int i = 0; i < dim; ++i) { t1 += lam[i] * C[i]; sq += C[i] * C[i]; }
        S.jE[j] = t1 + 0.5 * mu * sq;
    }
    if (!full) return;
    double* F = S.jF + 6 * j;
    for (int i = 0; i < 6; ++i) F[i] = 0.0;
    if (t == NXD_JOINT_ANGLE_LIMIT) {
        for (int i = 0; i < 2; ++i) F[i] = C[i] > 0.0 ? lam[i] + mu * C[i] : 0.0;
        S.jact[j] = (C[0] > 0.0 ? 1 : 0) | (C[1] > 0.0 ? 2 : 0);
    } else {
        for (int i = 0; i < dim; ++i) F[i] = mu * C[i] + lam[i];
        S.jact[j] = 0;
    }
    double* Jd = S.jJ + 72 * j;
    for (int r = 0; r < 6; ++r) for (int c = 0; c < 12; ++c) Jd[12 * r + c] = Jm[r][c];
}
__device__ __forceinline__ int joint_dim(int t) {
    return t == NXD_JOINT_HINGE || t == NXD_JOINT_FIXED ? 6 : (t == NXD_JOINT_SPHERICAL ? 3 : 2);
}
__device__ __forceinline__ bool joint_couples(const Solver& S, int j) {
    const int t = S.jtype[j];
    if (t == NXD_JOINT_FIXED) return false;
    if (t == NXD_JOINT_ANGLE_LIMIT) return S.jact[j] != 0;
    return true;
}

// DistanceBarrierForm::contactDistance (DistanceBarrierForm.cpp:88-99)
__device__ __forceinline__ double contact_distance(const ContactRec& c, const double* x) {
    const V3 pA = xs3(x, 6 * c.body_a), pB = xs3(x, 6 * c.body_b);
    return dmax(1e-9, dot(pB - pA, ld3(c.normal)));
}

__device__ void barrier_eval(const Solver& S, int c, const double* x) {
    const ContactRec& cr = S.contacts[c];
    const double dh = *S.bdhat_ptr, k = *S.bkappa_ptr;
    const double d = contact_distance(cr, x);
    S.bD[c] = d;
    S.bE[c] = barrier_value(d, dh, k);
    S.bGP[c] = d < dh ? barrier_gradient(d, dh, k) : 0.0;
    S.bHP[c] = d < dh ? barrier_hessian(d, dh, k) : 0.0;
}

// FrictionForm (FrictionForm.cpp:22-224) pieces at x
struct FricGeom { V3 rA, rB, n; double P[9]; };
__device__ void fric_geom(const Solver& S, const ContactRec& c, FricGeom& G) {
    const Q q0A = ldq(S.quat0 + 4 * c.body_a), q0B = ldq(S.quat0 + 4 * c.body_b);
    const Q rotA = ldq(S.qg + 4 * c.body_a), rotB = ldq(S.qg + 4 * c.body_b);
    const V3 pt = ld3(c.point);
    const V3 lA = qrot(qconj(q0A), pt - ld3(S.pos0 + 3 * c.body_a));
    const V3 lB = qrot(qconj(q0B), pt - ld3(S.pos0 + 3 * c.body_b));
    G.rA = qrot(rotA, lA);
    G.rB = qrot(rotB, lB);
    const V3 n = ld3(c.normal);
    G.n = sqnorm(n) > 1e-16 ? normalized(n) : v3(0, 1, 0);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) G.P[3 * i + j] = (i == j ? 1.0 : 0.0) - get(G.n, i) * get(G.n, j);
}
__device__ V3 fric_tangent(const Solver& S, const ContactRec& c, const FricGeom& G, const double* x, double dt) {
    const V3 dA = xs3(x, 6 * c.body_a) - ld3(S.pos0 + 3 * c.body_a);
    const V3 dB = xs3(x, 6 * c.body_b) - ld3(S.pos0 + 3 * c.body_b);
    V3 oA = v3(0, 0, 0), oB = v3(0, 0, 0), vA = v3(0, 0, 0), vB = v3(0, 0, 0);
    if (dt > 1e-12) {
        oA = xs3(x, 6 * c.body_a + 3) / dt; oB = xs3(x, 6 * c.body_b + 3) / dt;
        vA = dA / dt; vB = dB / dt;
    }
    vA = vA + cross(oA, G.rA);
    vB = vB + cross(oB, G.rB);
    const V3 rel = vB - vA;
    const V3 tv = rel - dot(rel, G.n) * G.n;
    return tv * dt;
}
__device__ void friction_eval(const Solver& S, int c, const double* x, bool full) {
    const int nnf = *S.nnf_ptr;
    const double N = c < nnf ? S.nforce[c] : 0.0;
    if (!(c < nnf) || N <= 0) { S.fE[c] = 0.0; return; }
    const ContactRec& cr = S.contacts[c];
    const double dt = *S.dt_ptr;
    FricGeom G;
    fric_geom(S, cr, G);
    const V3 u = fric_tangent(S, cr, G, x, dt);
    const double mu = S.friction_mu, eps = S.friction_eps;
    // FrictionPotential (Friction.cpp:5-61)
    const double un = norm(u);
    const double sn = sqrt(un * un + eps * eps);
    S.fE[c] = mu * N * (sn - eps);
    if (!full) return;
    V3 fg = v3(0, 0, 0);
    double Hf[9];
    if (un < 1e-12) {
        const double s = mu * N / eps;
        for (int i = 0; i < 9; ++i) Hf[i] = (i % 4 == 0) ? s : 0.0;
    } else {
        const double sc = mu * N / sn;
        fg = sc * u;
        const double s2 = sn * sn;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) Hf[3 * i + j] = sc * ((i == j ? 1.0 : 0.0) - get(u, i) * get(u, j) / s2);
    }
    st3(S.fFG + 3 * c, fg);
    for (int i = 0; i < 9; ++i) S.fHF[9 * c + i] = Hf[i];
    // J_A = [-P, P [rA]x], J_B = [P, -P [rB]x]
    M3 P;
    for (int i = 0; i < 9; ++i) P.m[i] = G.P[i];
    const M3 PA = mat_mul(P, cross_mat(G.rA)), PB = mat_mul(P, cross_mat(G.rB));
    double* JA = S.fJA + 18 * c;
    double* JB = S.fJB + 18 * c;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            JA[6 * i + j] = -G.P[3 * i + j]; JB[6 * i + j] = G.P[3 * i + j];
            JA[6 * i + 3 + j] = at(PA, i, j); JB[6 * i + 3 + j] = -at(PB, i, j);
        }
}

// VelocityDriveForm (VelocityDriveForm.cpp:61-417), stateful joint velocity.
__device__ double drive_target(const Drv& p, double filt) { return p.tau <= 0.0 ? p.vt : filt; }
__device__ double drive_dead(const Drv& p, double e) {
    if (p.delay <= 0.0) return e;
    if (e > p.delay) return e - p.delay;
    if (e < -p.delay) return e + p.delay;
    return 0.0;
}
__device__ double drive_sat(const Drv& p, double e) {
    const double raw = p.kv * e;
    if (!isfinite(p.maxT)) return raw;
    if (p.maxT <= 0.0) return raw;
    return p.maxT * nxm::tanh(raw / p.maxT);
}
__device__ double drive_velocity(const Solver& S, int d, const double* x) {
    const int A = S.da[d], B = S.db[d];
    const V3 tA = A >= 0 ? xs3(x, 6 * A + 3) : v3(0, 0, 0);
    const V3 tB = B >= 0 ? xs3(x, 6 * B + 3) : v3(0, 0, 0);
    const double dt = *S.dt_ptr;
    V3 oA = v3(0, 0, 0), oB = v3(0, 0, 0);
    if (S.dhas_prev[d]) {
        if (A >= 0) oA = dt <= 0 ? v3(0, 0, 0) : (tA - ld3(S.dprevA + 3 * d)) / dt;
        if (B >= 0) oB = dt <= 0 ? v3(0, 0, 0) : (tB - ld3(S.dprevB + 3 * d)) / dt;
    }
    const Drv& p = S.dprm[d];
    const double v = dot(oB - oA, v3(p.ax, p.ay, p.az));
    st3(S.dprevA + 3 * d, tA);
    st3(S.dprevB + 3 * d, tB);
    S.dhas_prev[d] = 1;
    return v;
}
// mode 0 value, 1 gradient, 2 hessian (stateful as in the reference)
__device__ void drive_eval(const Solver& S, int d, const double* x, int mode) {
    const Drv& p = S.dprm[d];
    const double dt = *S.dt_ptr;
    const double tgt = drive_target(p, S.dfilt[d]);
    if (mode == 0) {
        const double v = drive_velocity(S, d, x);
        const double e = drive_dead(p, tgt - v);
        double val;
        if (!isfinite(p.maxT)) val = 0.5 * p.kv * e * e;
        else if (p.kv <= 0.0 || p.maxT <= 0.0) val = 0.0;
        else { const double s = (p.kv * e) / p.maxT; val = (p.maxT * p.maxT / p.kv) * nxm::log(nxm::cosh(s)); }
        S.dE[d] = val;
    } else if (mode == 1) {
        const double v = drive_velocity(S, d, x);
        const double e = drive_dead(p, tgt - v);
        const double tq = drive_sat(p, e);
        S.dG[d] = dt <= 0 ? 0.0 : (-tq) * (1.0 / dt);
    } else {
        double H = dt <= 0 ? 0.0 : p.kv / (dt * dt);
        if (dt > 0 && isfinite(p.maxT) && p.kv > 0.0 && p.maxT > 0.0) {
            const double v = drive_velocity(S, d, x);
            const double e = tgt - v;
            if (fabs(e) <= p.delay) H = 0.0;
            else {
                const double ee = drive_dead(p, e);
                const double s = (p.kv * ee) / p.maxT;
                const double th = nxm::tanh(s);
                H = (p.kv * (1.0 - th * th)) / (dt * dt);
            }
        }
        S.dH[d] = H;
    }
}

// poses at x for every body (joint-style and friction-style rotations)
__device__ void eval_poses(const Solver& S, const double* x) {
    for (int i = threadIdx.x; i < S.N; i += blockDim.x) {
        const Q q0 = ldq(S.quat0 + 4 * i);
        const V3 th = xs3(x, 6 * i + 3);
        stq(S.qj + 4 * i, rot_joint(q0, th));
        stq(S.qg + 4 * i, rot_gt(q0, th));
    }
}

// ---------------------------------------------------------------------------
// Energies (computeValue / computeContactValue) at x
// ---------------------------------------------------------------------------
__device__ double energy_total(const Solver& S, const double* x, double s, int C, bool contact_only) {
    eval_poses(S, x);
    __syncthreads();
    const bool bar = *S.barrier_in_forms_ptr != 0, fr = *S.friction_form_ptr != 0;
    if (!contact_only) {
        for (int j = threadIdx.x; j < S.J; j += blockDim.x) joint_eval(S, j, x, false);
        for (int d = threadIdx.x; d < S.D; d += blockDim.x) drive_eval(S, d, x, 0);
    }
    for (int c = threadIdx.x; c < C; c += blockDim.x) {
        if (bar) barrier_eval(S, c, x);
        if (fr) friction_eval(S, c, x, false);
    }
    __syncthreads();
    double v = 0.0;
    if (!contact_only) {
        for (int i = threadIdx.x; i < S.N; i += blockDim.x) {
            const V3 dp = xs3(x, 6 * i) - xs3(S.xhat, 6 * i);
            const double et = 0.5 * S.mass[i] * sqnorm(dp);
            const V3 dth = xs3(x, 6 * i + 3) - xs3(S.xhat, 6 * i + 3);
            const double* I = S.inertia + 9 * i;
            const V3 r = v3(dth.x * I[0] + dth.y * I[3] + dth.z * I[6], dth.x * I[1] + dth.y * I[4] + dth.z * I[7],
                            dth.x * I[2] + dth.y * I[5] + dth.z * I[8]);
            S.red[i] = et + 0.5 * dot(r, dth);
        }
        const double inert = block_tree_sum(S.red, S.N);
        for (int i = threadIdx.x; i < S.N; i += blockDim.x)
            S.red[i] = -(S.mass[i] * dot(v3(0.0, -9.81, 0.0), xs3(x, 6 * i)));
        const double grav = block_tree_sum(S.red, S.N);
        for (int j = threadIdx.x; j < S.J; j += blockDim.x) S.red[j] = S.jE[j];
        const double cons = block_tree_sum(S.red, S.J);
        v = inert;
        v += s * grav;
        v += cons;
        for (int d = 0; d < S.D; ++d) v += s * S.dE[d];
    }
    if (bar) {
        for (int c = threadIdx.x; c < C; c += blockDim.x) S.red[c] = S.bE[c];
        v += s * block_tree_sum(S.red, C);
    }
    if (fr) {
        for (int c = threadIdx.x; c < C; c += blockDim.x) S.red[c] = S.fE[c];
        v += s * block_tree_sum(S.red, C);
    }
    return v;
}

// ---------------------------------------------------------------------------
// Gradient gather per body (item order), plus the contact-only gradient
// ---------------------------------------------------------------------------
__device__ void gather_gradient(const Solver& S, const double* x, double s, int C) {
    const bool bar = *S.barrier_in_forms_ptr != 0, fr = *S.friction_form_ptr != 0;
    const double dh = *S.bdhat_ptr;
    const int nnf = *S.nnf_ptr;
    for (int i = threadIdx.x; i < S.N; i += blockDim.x) {
        double g[6], t[6];
        const double m = S.mass[i];
        const V3 gp = m * (xs3(x, 6 * i) - xs3(S.xhat, 6 * i));
        const V3 gr = mat_vec(S.inertia + 9 * i, xs3(x, 6 * i + 3) - xs3(S.xhat, 6 * i + 3));
        g[0] = 0.0 + gp.x; g[1] = 0.0 + gp.y; g[2] = 0.0 + gp.z;
        g[3] = 0.0 + gr.x; g[4] = 0.0 + gr.y; g[5] = 0.0 + gr.z;
        const V3 fgv = -m * v3(0.0, -9.81, 0.0);
        g[0] += s * fgv.x; g[1] += s * fgv.y; g[2] += s * fgv.z;
        g[3] += s * 0.0; g[4] += s * 0.0; g[5] += s * 0.0;
        // ConstraintForm: J^T (mu C + lambda), joints in order
        for (int k = 0; k < 6; ++k) t[k] = 0.0;
        for (int q = S.jinc_off[i]; q < S.jinc_off[i + 1]; ++q) {
            const int j = S.jinc[q] >> 1, side = S.jinc[q] & 1;
            const int dim = joint_dim(S.jtype[j]);
            const double* Jd = S.jJ + 72 * j;
            const double* F = S.jF + 6 * j;
            for (int k = 0; k < 6; ++k) {
                double a = 0.0;
                for (int r = 0; r < dim; ++r) a += Jd[12 * r + 6 * side + k] * F[r];
                t[k] += a;
            }
        }
        for (int k = 0; k < 6; ++k) g[k] += t[k];
        // drives, each its own form
        for (int q = S.dinc_off[i]; q < S.dinc_off[i + 1]; ++q) {
            const int d = S.dinc[q] >> 1, side = S.dinc[q] & 1;
            const Drv& p = S.dprm[d];
            const double dEdq = S.dG[d];
            const V3 ax = v3(p.ax, p.ay, p.az);
            for (int k = 0; k < 3; ++k) {
                const double c = dEdq * get(ax, k);
                const double tk = side == 1 ? 0.0 + c : 0.0 - c;
                g[3 + k] += s * tk;
            }
            for (int k = 0; k < 3; ++k) g[k] += s * 0.0;
        }
        double cb[6] = {0, 0, 0, 0, 0, 0}, cf[6] = {0, 0, 0, 0, 0, 0};
        if (bar || fr) {
            for (int q = S.cinc_off[i]; q < S.cinc_off[i + 1]; ++q) {
                const int c = S.cinc[q] >> 1, side = S.cinc[q] & 1;
                const ContactRec& cr = S.contacts[c];
                if (bar && S.bD[c] < dh) {
                    const double gpv = S.bGP[c];
                    const V3 n = ld3(cr.normal);
                    const V3 contrib = side == 0 ? (-gpv) * n : gpv * n;
                    cb[0] += contrib.x; cb[1] += contrib.y; cb[2] += contrib.z;
                }
                if (fr && c < nnf && S.nforce[c] > 0) {
                    const double* Jx = (side == 0 ? S.fJA : S.fJB) + 18 * c;
                    const V3 fg = ld3(S.fFG + 3 * c);
                    for (int k = 0; k < 6; ++k) cf[k] += Jx[k] * fg.x + Jx[6 + k] * fg.y + Jx[12 + k] * fg.z;
                }
            }
        }
        double cgv[6];
        for (int k = 0; k < 6; ++k) cgv[k] = 0.0;
        if (bar) for (int k = 0; k < 6; ++k) { g[k] += s * cb[k]; cgv[k] += s * cb[k]; }
        if (fr) for (int k = 0; k < 6; ++k) { g[k] += s * cf[k]; cgv[k] += s * cf[k]; }
        for (int k = 0; k < 6; ++k) { S.g[6 * i + k] = g[k]; S.cg[6 * i + k] = cgv[k]; }
    }
}

// ---------------------------------------------------------------------------
// Hessian: diagonal block per body, coupling blocks per item
// ---------------------------------------------------------------------------
// 6x6 block contribution of a base joint to rows of side ra and cols of side ca
__device__ void joint_block(const Solver& S, int j, int ra, int ca, double* out) {
    const int dim = joint_dim(S.jtype[j]);
    const double* Jd = S.jJ + 72 * j;
    const double mu = S.jmu[j];
    for (int a = 0; a < 6; ++a)
        for (int b = 0; b < 6; ++b) {
            double sacc = 0.0;
            for (int r = 0; r < dim; ++r) sacc += Jd[12 * r + 6 * ra + a] * Jd[12 * r + 6 * ca + b];
            out[6 * a + b] = sacc * mu;
        }
}
__device__ void angle_limit_H(const Solver& S, int j, double* H3) {
    const double* ax = S.jparams + 16 * j;
    const double mu = S.jmu[j];
    for (int i = 0; i < 9; ++i) H3[i] = 0.0;
    for (int rep = 0; rep < 2; ++rep)
        if (S.jact[j] & (1 << rep))
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) H3[3 * a + b] += mu * (ax[a] * ax[b]);
}
// friction block J_X^T Hf J_Y, evaluated (J_X^T Hf) J_Y
__device__ void friction_block(const Solver& S, int c, int sx, int sy, double* out) {
    const double* Jx = (sx == 0 ? S.fJA : S.fJB) + 18 * c;
    const double* Jy = (sy == 0 ? S.fJA : S.fJB) + 18 * c;
    const double* Hf = S.fHF + 9 * c;
    for (int r = 0; r < 6; ++r) {
        const double T0 = Jx[r] * Hf[0] + Jx[6 + r] * Hf[3] + Jx[12 + r] * Hf[6];
        const double T1 = Jx[r] * Hf[1] + Jx[6 + r] * Hf[4] + Jx[12 + r] * Hf[7];
        const double T2 = Jx[r] * Hf[2] + Jx[6 + r] * Hf[5] + Jx[12 + r] * Hf[8];
        for (int cc = 0; cc < 6; ++cc) out[6 * r + cc] = T0 * Jy[cc] + T1 * Jy[6 + cc] + T2 * Jy[12 + cc];
    }
}

__device__ void gather_diag_hessian(const Solver& S, double s, int C) {
    const bool bar = *S.barrier_in_forms_ptr != 0, fr = *S.friction_form_ptr != 0;
    const double dh = *S.bdhat_ptr;
    const int nnf = *S.nnf_ptr;
    for (int i = threadIdx.x; i < S.N; i += blockDim.x) {
        double H[36];
        for (int k = 0; k < 36; ++k) H[k] = 0.0;
        const double m = S.mass[i];
        H[0] += m; H[7] += m; H[14] += m;
        for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) H[6 * (3 + a) + 3 + b] += S.inertia[9 * i + 3 * a + b];
        double blk[36];
        for (int q = S.jinc_off[i]; q < S.jinc_off[i + 1]; ++q) {
            const int j = S.jinc[q] >> 1, side = S.jinc[q] & 1;
            if (S.jtype[j] == NXD_JOINT_ANGLE_LIMIT) {
                if (!S.jact[j]) continue;
                double H3[9];
                angle_limit_H(S, j, H3);
                for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) H[6 * (3 + a) + 3 + b] += H3[3 * a + b];
            } else {
                joint_block(S, j, side, side, blk);
                for (int k = 0; k < 36; ++k) H[k] += blk[k];
            }
        }
        for (int q = S.dinc_off[i]; q < S.dinc_off[i + 1]; ++q) {
            const int d = S.dinc[q] >> 1;
            const double Hd = S.dH[d];
            if (Hd == 0.0) continue;
            const Drv& p = S.dprm[d];
            const double ax[3] = {p.ax, p.ay, p.az};
            for (int a = 0; a < 3; ++a) H[6 * (3 + a) + 3 + a] += (Hd * ax[a] * ax[a]) * s;
            for (int a = 0; a < 3; ++a)
                for (int b = a + 1; b < 3; ++b) {
                    const double od = Hd * ax[a] * ax[b];
                    H[6 * (3 + a) + 3 + b] += od * s;
                    H[6 * (3 + b) + 3 + a] += od * s;
                }
        }
        if (bar || fr) {
            for (int q = S.cinc_off[i]; q < S.cinc_off[i + 1]; ++q) {
                const int c = S.cinc[q] >> 1;
                if (!bar || !(S.bD[c] < dh)) continue;
                const double hp = S.bHP[c];
                const V3 n = ld3(S.contacts[c].normal);
                for (int r = 0; r < 3; ++r)
                    for (int cc = 0; cc < 3; ++cc) H[6 * r + cc] += (hp * (get(n, r) * get(n, cc))) * s;
            }
            for (int q = S.cinc_off[i]; q < S.cinc_off[i + 1]; ++q) {
                const int c = S.cinc[q] >> 1, side = S.cinc[q] & 1;
                if (!fr || !(c < nnf && S.nforce[c] > 0)) continue;
                friction_block(S, c, side, side, blk);
                for (int k = 0; k < 36; ++k) H[k] += blk[k] * s;
            }
        }
        for (int k = 0; k < 36; ++k) S.Hd[36 * i + k] = H[k];
    }
}

// Coupling block of item `it` with rows of body R and cols of body Cb (R != Cb),
// added into out (6x6, row-major).  Items: [0,J) joints, [J, J+C) barrier
// contacts, [J+C, J+2C) friction contacts.
__device__ void add_coupling_block(const Solver& S, int it, int R, int Cb, double s, double* out) {
    double blk[36];
    if (it < S.J) {
        const int j = it;
        const int ra = S.ja[j] == R ? 0 : 1, ca = S.ja[j] == Cb ? 0 : 1;
        if (S.jtype[j] == NXD_JOINT_ANGLE_LIMIT) {
            double H3[9];
            angle_limit_H(S, j, H3);
            for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) out[6 * (3 + a) + 3 + b] += -H3[3 * a + b];
        } else {
            joint_block(S, j, ra, ca, blk);
            for (int k = 0; k < 36; ++k) out[k] += blk[k];
        }
        return;
    }
    const int C = *S.ncontacts_ptr;
    if (it < S.J + C) {
        const int c = it - S.J;
        const double hp = S.bHP[c];
        const V3 n = ld3(S.contacts[c].normal);
        for (int r = 0; r < 3; ++r)
            for (int cc = 0; cc < 3; ++cc) out[6 * r + cc] += (-(hp * (get(n, r) * get(n, cc)))) * s;
        return;
    }
    const int c = it - S.J - C;
    const int sx = S.contacts[c].body_a == R ? 0 : 1, sy = S.contacts[c].body_a == Cb ? 0 : 1;
    friction_block(S, c, sx, sy, blk);
    for (int k = 0; k < 36; ++k) out[k] += blk[k] * s;
}
__device__ __forceinline__ void item_bodies(const Solver& S, int it, int& a, int& b) {
    if (it < S.J) { a = S.ja[it]; b = S.jb[it]; return; }
    const int C = *S.ncontacts_ptr;
    const int c = it < S.J + C ? it - S.J : it - S.J - C;
    a = S.contacts[c].body_a; b = S.contacts[c].body_b;
}
__device__ __forceinline__ bool item_active(const Solver& S, int it) {
    if (it < S.J) return joint_couples(S, it);
    const int C = *S.ncontacts_ptr;
    if (it < S.J + C) return *S.barrier_in_forms_ptr != 0 && S.bD[it - S.J] < *S.bdhat_ptr;
    const int c = it - S.J - C;
    return *S.friction_form_ptr != 0 && c < *S.nnf_ptr && S.nforce[c] > 0;
}

// ---------------------------------------------------------------------------
// Union-find (concurrent, root = smallest body index of the component)
// ---------------------------------------------------------------------------
__device__ int uf_find(int* par, int x) {
    // parents only ever point to smaller roots, so a chain is shorter than N;
    // the bound only guards against corrupted input
    for (int it = 0; it < (1 << 24); ++it) {
        const int p = par[x];
        if (p == x) return x;
        x = p;
    }
    return x;
}
__device__ void uf_union(int* par, int a, int b) {
    for (int it = 0; it < 1 << 20; ++it) {
        a = uf_find(par, a);
        b = uf_find(par, b);
        if (a == b) return;
        if (a < b) { const int t = a; a = b; b = t; }
        // hook root a (larger) under b
        if (atomicCAS(&par[a], a, b) == a) return;
    }
}

// stable bucket placement, warp 0, entries e in [0, n): key(e) -> out position
// offs[key] holds the running start per key (already the exclusive scan).
template <typename KeyFn>
__device__ void warp_stable_place(int n, KeyFn key, int* offs, int* out) {
    if (threadIdx.x >= 32) return;
    const int lane = threadIdx.x;
    const unsigned lt = (1u << lane) - 1u;
    for (int base = 0; base < n; base += 32) {
        const int e = base + lane;
        const bool valid = e < n;
        const int k = valid ? key(e) : -1 - lane;
        const unsigned mask = __match_any_sync(0xffffffffu, k);
        const int rank = __popc(mask & lt);
        int start = 0;
        if (valid) start = offs[k];
        __syncwarp();
        if (valid) out[start + rank] = e;
        const int leader = __ffs(mask) - 1;
        if (valid && lane == leader) offs[k] = start + __popc(mask);
        __syncwarp();
    }
}

}  // namespace nx

namespace nx {

// LDL^T of one 6x6 block (lower part of H), left-looking exactly as the dense
// oracle loop; solves rhs in place.  Returns false on a zero pivot.
__device__ bool ldlt6_solve(double* A, double* b) {
    double d[6];
    for (int j = 0; j < 6; ++j) {
        double dj = A[6 * j + j];
        for (int k = 0; k < j; ++k) { const double l = A[6 * j + k]; dj -= l * l * d[k]; }
        if (dj == 0.0) return false;
        d[j] = dj;
        A[6 * j + j] = dj;
        for (int i = j + 1; i < 6; ++i) {
            double s = A[6 * i + j];
            for (int k = 0; k < j; ++k) s -= A[6 * i + k] * A[6 * j + k] * d[k];
            A[6 * i + j] = s / dj;
        }
    }
    for (int i = 0; i < 6; ++i) { double s = b[i]; for (int k = 0; k < i; ++k) s -= A[6 * i + k] * b[k]; b[i] = s; }
    for (int i = 0; i < 6; ++i) b[i] /= A[6 * i + i];
    for (int i = 5; i >= 0; --i) { double s = b[i]; for (int k = 5; k > i; --k) s -= A[6 * k + i] * b[k]; b[i] = s; }
    return true;
}

__device__ __forceinline__ void tri_index(int t, int& a, int& b) {
    int r = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((r + 1) * (r + 2) / 2 <= t) ++r;
    while (r * (r + 1) / 2 > t) --r;
    a = r;
    b = t - r * (r + 1) / 2;
}

// Warp-level block-skipping right-looking LDL^T + solve of one component
// matrix A (n x n row-major, lower part valid), nzb (k x k, lower, with fill).
__device__ bool warp_ldlt_solve(double* A, int n, int k, const unsigned char* nzb, int* cand, double* dpiv, double* rhs) {
    const int lane = threadIdx.x & 31;
    bool ok = true;
    for (int j = 0; j < n; ++j) {
        const int bj = j / 6;
        int m = 0;
        for (int i = j + 1; i < 6 * bj + 6; ++i) { if (lane == 0) cand[m] = i; ++m; }
        for (int bi = bj + 1; bi < k; ++bi)
            if (nzb[(size_t)bi * k + bj]) { if (lane < 6) cand[m + lane] = 6 * bi + lane; m += 6; }
        __syncwarp();
        const double dj = A[(size_t)j * n + j];
        if (dj == 0.0) { ok = false; break; }
        for (int t = lane; t < m; t += 32) { const int i = cand[t]; A[(size_t)i * n + j] = A[(size_t)i * n + j] / dj; }
        __syncwarp();
        const int np = m * (m + 1) / 2;
        for (int t = lane; t < np; t += 32) {
            int a, b;
            tri_index(t, a, b);
            const int i = cand[a], c = cand[b];
            A[(size_t)i * n + c] -= (A[(size_t)i * n + j] * A[(size_t)c * n + j]) * dj;
        }
        if (lane == 0) dpiv[j] = dj;
        __syncwarp();
    }
    if (!ok) return false;
    for (int j = 0; j < n; ++j) {
        const int bj = j / 6;
        const double yj = rhs[j];
        for (int i = j + 1 + lane; i < 6 * bj + 6; i += 32) rhs[i] -= A[(size_t)i * n + j] * yj;
        for (int bi = bj + 1; bi < k; ++bi)
            if (nzb[(size_t)bi * k + bj] && lane < 6) { const int i = 6 * bi + lane; rhs[i] -= A[(size_t)i * n + j] * yj; }
        __syncwarp();
    }
    for (int i = lane; i < n; i += 32) rhs[i] /= dpiv[i];
    __syncwarp();
    for (int j = n - 1; j >= 0; --j) {
        const int bj = j / 6;
        const double xj = rhs[j];
        for (int i = 6 * bj + lane; i < j; i += 32) rhs[i] -= A[(size_t)j * n + i] * xj;
        for (int bc = 0; bc < bj; ++bc)
            if (nzb[(size_t)bj * k + bc] && lane < 6) { const int i = 6 * bc + lane; rhs[i] -= A[(size_t)j * n + i] * xj; }
        __syncwarp();
    }
    return true;
}

// Solve H dx = -g.  Returns false (all threads) on failure.
__device__ bool solve_newton_system(const Solver& S, double s, int C, int* sh_flag) {
    const int N = S.N;
    const int n_items = S.J + 2 * C;
    // union-find
    for (int i = threadIdx.x; i < N; i += blockDim.x) S.parent[i] = i;
    if (threadIdx.x == 0) *sh_flag = 0;
    __syncthreads();
    for (int it = threadIdx.x; it < n_items; it += blockDim.x) {
        if (!item_active(S, it)) continue;
        int a, b;
        item_bodies(S, it, a, b);
        if (a != b) uf_union(S.parent, a, b);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < N; i += blockDim.x) S.comp[i] = uf_find(S.parent, i);
    __syncthreads();
    // component sizes (indexed by root) and member lists (bodies ascending)
    for (int i = threadIdx.x; i < N; i += blockDim.x) S.comp_size[i] = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < N; i += blockDim.x) atomicAdd(&S.comp_size[S.comp[i]], 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int r = 0; r < N; ++r) { S.comp_off[r] = acc; acc += S.comp_size[r]; }
        S.comp_off[N] = acc;
        *S.pool_off = 0;
        *S.nzb_off = 0;
    }
    __syncthreads();
    // running starts live in item_comp_off temporarily for the placement
    for (int r = threadIdx.x; r <= N; r += blockDim.x) S.item_comp_off[r] = S.comp_off[r];
    __syncthreads();
    warp_stable_place(N, [&](int e) { return S.comp[e]; }, S.item_comp_off, S.members);
    __syncthreads();
    // active coupling items grouped by component root, item order kept
    for (int r = threadIdx.x; r <= N; r += blockDim.x) S.deg[r] = 0;
    __syncthreads();
    for (int it = threadIdx.x; it < n_items; it += blockDim.x) {
        S.items[it] = -1;
        if (!item_active(S, it)) continue;
        int a, b;
        item_bodies(S, it, a, b);
        if (a == b) continue;
        S.items[it] = S.comp[a];
        atomicAdd(&S.deg[S.comp[a]], 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int r = 0; r < N; ++r) { const int c = S.deg[r]; S.deg[r] = acc; acc += c; }
        S.deg[N] = acc;
        *S.n_items_ptr = acc;
    }
    __syncthreads();
    for (int r = threadIdx.x; r <= N; r += blockDim.x) S.item_comp_off[r] = S.deg[r];
    __syncthreads();
    {
        // compact active items in order, then stable-place by component
        // (items[] holds the component root or -1)
        if (threadIdx.x < 32) {
            const int lane = threadIdx.x;
            const unsigned lt = (1u << lane) - 1u;
            for (int base = 0; base < n_items; base += 32) {
                const int e = base + lane;
                const int key = e < n_items ? S.items[e] : -1;
                const bool valid = key >= 0;
                const unsigned mask = __match_any_sync(0xffffffffu, valid ? key : -1 - lane);
                const int rank = __popc(mask & lt);
                int start = 0;
                if (valid) start = S.item_comp_off[key];
                __syncwarp();
                if (valid) S.item_list[start + rank] = e;
                const int leader = __ffs(mask) - 1;
                if (valid && lane == leader) S.item_comp_off[key] = start + __popc(mask);
                __syncwarp();
            }
        }
    }
    __syncthreads();
    // singletons: one thread each
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        if (S.comp[i] != i || S.comp_size[i] != 1) continue;
        double A[36], b[6];
        for (int k = 0; k < 36; ++k) A[k] = S.Hd[36 * i + k];
        for (int k = 0; k < 6; ++k) b[k] = -S.g[6 * i + k];
        if (!ldlt6_solve(A, b)) { atomicExch(sh_flag, 1); continue; }
        for (int k = 0; k < 6; ++k) S.dx[6 * i + k] = b[k];
    }
    // multi-body components: one warp each
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    int* cand = S.cand + (size_t)wid * S.cand_stride;
    int ci = 0;
    for (int r = 0; r < N; ++r) {
        if (S.comp_size[r] < 2 || S.comp[r] != r) continue;
        if ((ci++ % nw) != wid) continue;
        const int k = S.comp_size[r];
        const int* mem = S.members + S.comp_off[r];
        if (k > kMaxComponentBodies) { if (lane == 0) { atomicExch(sh_flag, 1); atomicExch(S.status, NXD_CAPACITY); } continue; }
        const int n = 6 * k;
        long long aoff = 0, zoff = 0;
        if (lane == 0) {
            aoff = atomicAdd((unsigned long long*)S.pool_off, (unsigned long long)n * n);
            zoff = atomicAdd((unsigned long long*)S.nzb_off, (unsigned long long)k * k);
        }
        aoff = __shfl_sync(0xffffffffu, aoff, 0);
        zoff = __shfl_sync(0xffffffffu, zoff, 0);
        if (aoff + (long long)n * n > S.pool_cap || zoff + (long long)k * k > S.nzb_cap) {
            if (lane == 0) { atomicExch(sh_flag, 1); atomicExch(S.status, NXD_CAPACITY); }
            continue;
        }
        double* A = S.pool + aoff;
        unsigned char* nz = S.nzb + zoff;
        const int i0 = S.deg[r], i1 = S.deg[r + 1];
        // provisional local index = rank in ascending member order
        for (int t = lane; t < k; t += 32) S.local[mem[t]] = t;
        for (int t = lane; t < k * k; t += 32) nz[t] = 0;
        __syncwarp();
        for (int q = i0 + lane; q < i1; q += 32) {
            int a, b;
            item_bodies(S, S.item_list[q], a, b);
            const int la = S.local[a], lb = S.local[b];
            nz[la * k + lb] = 1; nz[lb * k + la] = 1;
        }
        __syncwarp();
        // order members by (distinct neighbours, body index)
        int* ord = cand + 6 * kMaxComponentBodies;       // k ints
        int* dg = ord + kMaxComponentBodies;             // k ints
        for (int t = lane; t < k; t += 32) {
            int c = 0;
            for (int u = 0; u < k; ++u) c += (u != t && nz[t * k + u]) ? 1 : 0;
            dg[t] = c;
            ord[t] = mem[t];
        }
        __syncwarp();
        if (lane == 0) {
            for (int a = 1; a < k; ++a) {
                const int vb = ord[a], vd = dg[a];
                int b = a - 1;
                while (b >= 0 && (dg[b] > vd || (dg[b] == vd && ord[b] > vb))) { ord[b + 1] = ord[b]; dg[b + 1] = dg[b]; --b; }
                ord[b + 1] = vb; dg[b + 1] = vd;
            }
        }
        __syncwarp();
        for (int t = lane; t < k; t += 32) S.local[ord[t]] = t;
        for (int t = lane; t < k * k; t += 32) nz[t] = 0;
        __syncwarp();
        for (int q = i0 + lane; q < i1; q += 32) {
            int a, b;
            item_bodies(S, S.item_list[q], a, b);
            const int la = S.local[a], lb = S.local[b];
            nz[max(la, lb) * k + min(la, lb)] = 1;
        }
        __syncwarp();
        // symbolic fill, column by column
        for (int bj = 0; bj < k; ++bj) {
            for (int t = lane; t < k * k; t += 32) {
                const int b2 = t / k, b1 = t % k;
                if (b1 > bj && b2 > b1 && nz[(size_t)b1 * k + bj] && nz[(size_t)b2 * k + bj]) nz[(size_t)b2 * k + b1] = 1;
            }
            __syncwarp();
        }
        // zero used blocks, place diagonal blocks (lower part)
        for (int t = lane; t < k * k; t += 32) {
            const int bi = t / k, bc = t % k;
            if (bc > bi) continue;
            if (bc != bi && !nz[t]) continue;
            for (int e = 0; e < 36; ++e) {
                const int rr = e / 6, cc = e % 6;
                double v = 0.0;
                if (bc == bi && cc <= rr) v = S.Hd[36 * ord[bi] + e];
                A[(size_t)(6 * bi + rr) * n + 6 * bc + cc] = v;
            }
        }
        __syncwarp();
        // coupling items in item order, lower orientation in local order
        if (lane == 0) {
            for (int q = i0; q < i1; ++q) {
                const int it = S.item_list[q];
                int a, b;
                item_bodies(S, it, a, b);
                const int la = S.local[a], lb = S.local[b];
                const int R = la > lb ? a : b, Cb = la > lb ? b : a;
                const int lr = max(la, lb), lc = min(la, lb);
                double blk[36];
                for (int e = 0; e < 36; ++e) blk[e] = 0.0;
                add_coupling_block(S, it, R, Cb, s, blk);
                for (int e = 0; e < 36; ++e) A[(size_t)(6 * lr + e / 6) * n + 6 * lc + e % 6] += blk[e];
            }
        }
        __syncwarp();
        // rhs and pivots: the component's members own DOF range
        // [6 comp_off, 6 comp_off + n) of dvec ([12N] doubles)
        double* b = S.dvec + 6 * (size_t)S.comp_off[r];
        double* dp = S.dvec + 6 * (size_t)N + 6 * (size_t)S.comp_off[r];
        for (int t = lane; t < n; t += 32) b[t] = -S.g[6 * ord[t / 6] + t % 6];
        __syncwarp();
        if (!warp_ldlt_solve(A, n, k, nz, cand, dp, b)) { if (lane == 0) atomicExch(sh_flag, 1); continue; }
        for (int t = lane; t < n; t += 32) S.dx[6 * ord[t / 6] + t % 6] = b[t];
        __syncwarp();
    }
    __syncthreads();
    const bool fail = *sh_flag != 0;
    __syncthreads();
    return !fail;
}

// ---------------------------------------------------------------------------
// The kernel: one ALM iteration's Newton solve + joint bookkeeping.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kSolverThreads) k_newton(Solver S) {
    __shared__ double sh_red[32];
    __shared__ int sh_flag;
    __shared__ int sh_done;
    if (*S.alm_done) return;
    const int N = S.N;
    const int C = *S.ncontacts_ptr;
    const double dt = *S.dt_ptr;
    const double s = dt * dt;
    const int n6 = 6 * N;
    // contact incidence (body -> contact*2+side), contact order kept
    for (int i = threadIdx.x; i <= N; i += blockDim.x) S.cinc_cnt[i] = 0;
    __syncthreads();
    for (int e = threadIdx.x; e < 2 * C; e += blockDim.x) {
        const ContactRec& cr = S.contacts[e >> 1];
        atomicAdd(&S.cinc_cnt[(e & 1) ? cr.body_b : cr.body_a], 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int i = 0; i < N; ++i) { S.cinc_off[i] = acc; acc += S.cinc_cnt[i]; }
        S.cinc_off[N] = acc;
    }
    __syncthreads();
    for (int i = threadIdx.x; i <= N; i += blockDim.x) S.cinc_cnt[i] = S.cinc_off[i];
    __syncthreads();
    warp_stable_place(2 * C, [&](int e) { const ContactRec& cr = S.contacts[e >> 1]; return (e & 1) ? cr.body_b : cr.body_a; },
                      S.cinc_cnt, S.cinc);
    __syncthreads();

    bool converged = false;
    int iters = 0;
    for (int iter = 0; iter < S.newton_max_iters; ++iter) {
        iters = iter;
        // gradient at x (drives: gradient call)
        eval_poses(S, S.x);
        __syncthreads();
        for (int j = threadIdx.x; j < S.J; j += blockDim.x) joint_eval(S, j, S.x, true);
        for (int d = threadIdx.x; d < S.D; d += blockDim.x) drive_eval(S, d, S.x, 1);
        const bool bar = *S.barrier_in_forms_ptr != 0, fr = *S.friction_form_ptr != 0;
        for (int c = threadIdx.x; c < C; c += blockDim.x) {
            if (bar) barrier_eval(S, c, S.x);
            if (fr) friction_eval(S, c, S.x, true);
        }
        __syncthreads();
        gather_gradient(S, S.x, s, C);
        __syncthreads();
        double gm = 0.0;
        for (int k = threadIdx.x; k < n6; k += blockDim.x) gm = dmax(gm, fabs(S.g[k]));
        gm = block_max(gm, sh_red);
        if (gm < S.newton_tol) { converged = true; break; }
        // Hessian (drives: hessian call)
        for (int d = threadIdx.x; d < S.D; d += blockDim.x) drive_eval(S, d, S.x, 2);
        __syncthreads();
        gather_diag_hessian(S, s, C);
        __syncthreads();
        if (!solve_newton_system(S, s, C, &sh_flag)) break;
        // line search (max step 1)
        const double fx = energy_total(S, S.x, s, C, false);
        for (int k = threadIdx.x; k < n6; k += blockDim.x) S.red[k] = S.g[k] * S.dx[k];
        const double descent = block_tree_sum(S.red, n6);
        const double fc = energy_total(S, S.x, s, C, true);
        for (int k = threadIdx.x; k < n6; k += blockDim.x) S.red[k] = S.cg[k] * S.dx[k];
        const double cdesc = block_tree_sum(S.red, n6);
        if (descent > 0) { if (threadIdx.x == 0) atomicAdd(S.ls_fail, 1); break; }
        double alpha = 1.0;
        if (threadIdx.x == 0) sh_done = 0;
        __syncthreads();
        for (int ls = 0; ls < S.ls_max_iters; ++ls) {
            for (int k = threadIdx.x; k < n6; k += blockDim.x) S.xt[k] = S.x[k] + alpha * S.dx[k];
            __syncthreads();
            const double fn = energy_total(S, S.xt, s, C, false);
            const double fcn = energy_total(S, S.xt, s, C, true);
            const bool cok = cdesc <= 0.0 ? (fcn <= fc + S.ls_c1 * alpha * cdesc) : (fcn <= fc);
            if (fn <= fx + S.ls_c1 * alpha * descent && cok) { sh_done = 1; break; }
            alpha *= S.ls_rho;
        }
        __syncthreads();
        if (!sh_done) { if (threadIdx.x == 0) atomicAdd(S.ls_fail, 1); break; }
        for (int k = threadIdx.x; k < n6; k += blockDim.x) S.x[k] = S.xt[k];
        __syncthreads();
        if (iter == S.newton_max_iters - 1) iters = S.newton_max_iters;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        atomicAdd(S.newton_iters, iters);
        *S.converged = converged ? 1 : 0;
    }
    // ALM: violation, hardening, lambda update (IPCSolver.cpp:1084-1110)
    eval_poses(S, S.x);
    __syncthreads();
    for (int j = threadIdx.x; j < S.J; j += blockDim.x) joint_eval(S, j, S.x, false);
    __syncthreads();
    if (threadIdx.x == 0) {
        double mcv = 0.0, dual = 0.0;
        for (int j = 0; j < S.J; ++j) {
            const int dim = joint_dim(S.jtype[j]);
            double inf = 0.0;
            for (int k = 0; k < dim; ++k) inf = dmax(inf, fabs(S.jC[6 * j + k]));
            mcv = dmax(mcv, inf);
            const double dc = S.jmu[j] * inf;
            if (isfinite(dc)) dual = dmax(dual, dmin(dc, 1e12));
            else dual = dmax(dual, 1e12);
            if (inf > S.alm_hardening_trigger * S.alm_constraint_tol) {
                const double ns = S.jmu[j] * S.alm_hardening_ratio;
                S.jmu[j] = isfinite(ns) ? dmin(ns, 1e12) : 1e12;
            }
        }
        *S.alm_mcv = mcv;
        *S.alm_dual = dual;
    }
    __syncthreads();
    for (int j = threadIdx.x; j < S.J; j += blockDim.x) {
        const int dim = joint_dim(S.jtype[j]);
        const double* Cj = S.jC + 6 * j;
        double* lam = S.jlam + 6 * j;
        const double mu = S.jmu[j];
        if (S.jtype[j] == NXD_JOINT_ANGLE_LIMIT) for (int k = 0; k < dim; ++k) lam[k] = dmax(0.0, lam[k] + mu * Cj[k]);
        else for (int k = 0; k < dim; ++k) lam[k] += mu * Cj[k];
    }
}

}  // namespace nx
