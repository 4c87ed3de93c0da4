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
//    ordered by (distinct coupled neighbours, body index); every entry of L
//    takes its updates (L_ik L_jk) d_k in ascending k over the structurally
//    nonzero k (left-looking), forward substitution subtracts in ascending and
//    backward substitution in descending column order.
#pragma once

#include "nx_math.cuh"
#include "geometry.cuh"

namespace nx {

// Optional per-phase cycle counters of k_newton (build with -DNXD_PHASE_TIMERS;
// thread 0 prints one line per launch).  Off in the product build.
#ifdef NXD_PHASE_TIMERS
__shared__ long long nx_ph_acc[8];
__shared__ long long nx_ph_last;
#define NX_PHASE_START() do { if (threadIdx.x == 0) { for (int q_ = 0; q_ < 8; ++q_) nx_ph_acc[q_] = 0; nx_ph_last = clock64(); } } while (0)
#define NX_PHASE(k) do { if (threadIdx.x == 0) { const long long t_ = clock64(); nx_ph_acc[k] += t_ - nx_ph_last; nx_ph_last = t_; } } while (0)
#else
#define NX_PHASE_START() do {} while (0)
#define NX_PHASE(k) do {} while (0)
#endif

constexpr int kSolverThreads = 1024;
constexpr int kMaxComponentBodies = 2048;   // structure masks of <= 64 words per row
constexpr int kMaxIncidence = 4096;          // 2 x kMaxContacts contact ends, sorted in shared memory
// A body with more contact ends than this (the hopper under a pile) has its
// per-DOF gradient and Hessian-row sums done by a warp: the lanes evaluate 32
// contacts' terms at a time and every lane adds them in contact order.
constexpr int kHeavyEnds = 32;
static_assert(2 * kMaxContacts <= kMaxIncidence, "contact incidence sort buffer too small");

// Control-form parameters (8 doubles, the nxd_scene_desc layout after the
// creation-time normalisation):
//   angular / linear velocity drive: axis, kv, v_target, max torque / force
//     (inf: unlimited), delay deadzone, delay filter time constant
//   position drive: axis, kp (kv), target position (vt), max force (maxT),
//     deadzone (delay)
//   force drive: force (ax, ay, az), torque (kv, vt, maxT)
//   damped spring: rest length (ax), stiffness (ay), damping (az)
struct Drv {
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
    const int* dkind;                             // [D] NXD_DRIVE_*
    double* dDir;                                 // [3D] spring direction of the last gradient / Hessian call
    const double* bvel;                           // [3N] body velocities of the step start (DampedSpringForm)
    // contacts
    const ContactRec* contacts; const int* ncontacts_ptr;
    const double* nforce; const int* nnf_ptr;
    int* cinc_off; int* cinc;                     // body -> contact*2+side, ascending; built per kernel
    int* heavy; int* heavy_list; int* n_heavy;    // bodies with more than kHeavyEnds contact ends (k_newton)
    // scalars
    const double* dt_ptr; const double* scale_ptr; const double* bdhat_ptr; const double* bkappa_ptr;
    const int* barrier_in_forms_ptr; const int* friction_form_ptr;
    const double* friction_mu_ptr;                // FrictionForm coefficient of the step
    double friction_eps;
    int newton_max_iters, ls_max_iters;
    double newton_tol, ls_c1, ls_rho;
    double alm_constraint_tol, alm_hardening_trigger, alm_hardening_ratio;
    // scratch
    double* g; double* cg; double* dx; double* xt;                 // [6N]
    double* qj; double* qg;                                        // [N*4] poses at the evaluation point
    double* jC; double* jF; double* jJ; double* jE; int* jact;     // joints (jJ: 6 x 12 per joint)
    double* bD; double* bGP; double* bHP; double* bE;               // barrier per contact
    double* fFG; double* fHF; double* fJA; double* fJB; double* fE; // friction per contact
    double* dE; double* dG; double* dH;                            // drives
    double* Hd;                                                    // [N*36] diagonal blocks
    // linear solve
    int* parent; int* comp;                       // [N] union-find parent, component root per body
    int* mcnt; int* icnt; int* rflag;             // [N+1] per root: members, coupling items, multi-body flag
    int* comp_root; int* n_comp; int* comp_next;  // multi-body components by ordinal; work counter
    int* members; int* items;                     // [N], [J+2C] grouped per component
    int* local;                                   // [N] body -> member index inside its component
    unsigned* mpool; long long mpool_cap; long long* mpool_off;   // per-component masks and lists
    double* pool; long long pool_cap; long long* pool_off;        // per-component L, D and rhs
    int slab_bytes;                               // per-warp shared workspace of a component solve (0: none)
    int* solve_fail;                              // [1] zero pivot or capacity in this solve
    int* iact;                                    // [J+D+2*Cmax] item active at the last structure build
    // external linear system (nxd_linear_solve): when ext_n >= 0 the coupling
    // items are the caller's BSR blocks (row, col, 36 values), diagonal
    // blocks inactive, instead of joints, control forms and contacts
    int ext_n; const int* ext_row; const int* ext_col; const double* ext_vals;
    // grid execution of k_newton
    unsigned* bar_count; int* bar_abort;          // barrier arrivals and give-up flag, zeroed per launch
    unsigned spin_limit;                          // polls before a barrier wait gives up (0: kBarrierSpinLimit)
    int dbg_hold;                                 // failure-detection hook: the last CTA stays away (bounded)
    double* gpart;                                // [2 * kRedMaxQ * kMaxNewtonGrid] per-CTA partial sums
    // outputs / state
    int* alm_done; int* status; int* newton_iters; int* converged; int* ls_fail;
    double* alm_mcv; double* alm_dual;
};

// ---------------------------------------------------------------------------
// Block-level helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ int pow2_ceil(int n) { int p = 1; while (p < n) p <<= 1; return p; }

// Block reductions.
//
// The fixed tree over n values pads to P = pow2 >= n with zeros and runs
// v[i] += v[i + h] for h = P/2 .. 1.  Padding further only adds exact zeros
// at the top levels, so take P >= the number of threads T.  After the levels
// with h >= nw (the warp count), v[w] is the same tree over the residue class
// {w + nw m}; inside that class, after its levels with stride >= 32 nw,
// element m = l + 32 j reduces to the tree over j of v[w + nw l + T j].  So
// warp w, lane l folds j (K = P / T values; the stride tree is the
// contiguous pairwise tree over the bit-reversed index, kept as a stack of
// partial sums), the lanes finish class w with shuffles (h = 16 .. 1), and
// the nw class sums go through shared memory once for the last levels.  The
// result is the same double as the plain loop, with one __syncthreads.
constexpr int kRedMaxQ = 8;

// Fold of the K = P / stride values f(base + stride * m), m < K (P = the
// padded length, a power of two >= stride), in stride-tree order: the
// contiguous pairwise tree over the bit-reversed m, kept as a stack of
// partial sums.  Elements at or past n are zero.
template <typename F>
__device__ __forceinline__ double lane_fold(int n, int base, int stride, F f) {
    const int P = max(pow2_ceil(max(n, 1)), stride);
    const int K = P / stride;
    if (K == 1) return base < n ? f(base) : 0.0;
    const int lg = 31 - __clz(K);
    double stk[24];
    int top = 0;
    for (int j = 0; j < K; ++j) {
        const int e = base + stride * (int)(__brev((unsigned)j) >> (32 - lg));
        double v = e < n ? f(e) : 0.0;
        for (int c = j + 1; !(c & 1); c >>= 1) v = stk[--top] + v;
        stk[top++] = v;
    }
    return stk[0];
}
__device__ __forceinline__ double warp_tree(double v) {
    for (int h = 16; h >= 1; h >>= 1) v = v + __shfl_down_sync(0xffffffffu, v, h);
    return __shfl_sync(0xffffffffu, v, 0);
}

// Reduction scratch of one CTA (blockDim a power of two >= 32, nw warps):
// warp w, lane l folds the elements w + nw l + blockDim j; two alternating
// buffers of class sums, so that a call's writes never meet the previous
// call's reads.
struct BlockRed {
    double* sh;      // 2 * kRedMaxQ * 32 doubles of shared memory
    int parity;
    template <int Q, typename F>
    __device__ void sums(const int (&n)[Q], F f, double (&out)[Q]) {
        static_assert(Q <= kRedMaxQ, "too many simultaneous reductions");
        const int B = blockDim.x, nw = B >> 5;
        const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
        double* buf = sh + parity * (kRedMaxQ * 32);
        parity ^= 1;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const double v = warp_tree(lane_fold(n[q], w + nw * l, B, [&](int e) { return f(q, e); }));
            if (l == 0) buf[q * 32 + w] = v;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < Q; ++q) out[q] = warp_tree(l < nw ? buf[q * 32 + l] : 0.0);
    }
    template <typename F>
    __device__ double sum(int n, F f) {
        const int nn[1] = {n};
        double o[1];
        sums<1>(nn, [&](int, int e) { return f(e); }, o);
        return o[0];
    }
    __device__ double max(double v) {
        for (int o = 16; o > 0; o >>= 1) v = dmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        double* buf = sh + parity * (kRedMaxQ * 32);
        parity ^= 1;
        if ((threadIdx.x & 31) == 0) buf[threadIdx.x >> 5] = v;
        __syncthreads();
        double w = (threadIdx.x & 31) < (blockDim.x >> 5) ? buf[threadIdx.x & 31] : 0.0;
        for (int o = 16; o > 0; o >>= 1) w = dmax(w, __shfl_xor_sync(0xffffffffu, w, o));
        return w;
    }
};
#define NX_BLOCK_RED(name)                                   \
    __shared__ double name##_buf[2 * kRedMaxQ * 32];         \
    BlockRed name;                                           \
    name.sh = name##_buf;                                    \
    name.parity = 0

// Exclusive prefix sums of Q int arrays of length n, in place allowed; a[n]
// receives the total.  Thread t of the CTA scans the chunk [t c, t c + c),
// c = ceil(n / blockDim).  sh: 32 Q ints.  The caller synchronises before
// reading the result.
template <int Q>
__device__ void block_scan_excl(int* const (&a)[Q], int n, int* sh) {
    const int t = threadIdx.x, lane = t & 31, w = t >> 5, nw = blockDim.x >> 5;
    const int c = (n + blockDim.x - 1) / blockDim.x;
    const int b0 = min(n, t * c), b1 = min(n, b0 + c);
    int v[Q], incl[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        int acc = 0;
        for (int i = b0; i < b1; ++i) acc += a[q][i];
        v[q] = acc;
        int x = acc;
        for (int o = 1; o < 32; o <<= 1) { const int y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
        incl[q] = x;
        if (lane == 31) sh[q * 32 + w] = x;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        int x = lane < nw ? sh[q * 32 + lane] : 0;
        for (int o = 1; o < 32; o <<= 1) { const int y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
        const int prev = __shfl_sync(0xffffffffu, x, (w + 31) & 31);
        const int wbase = w > 0 ? prev : 0;
        const int total = __shfl_sync(0xffffffffu, x, 31);
        int run = wbase + incl[q] - v[q];
        for (int i = b0; i < b1; ++i) { const int e = a[q][i]; a[q][i] = run; run += e; }
        if (t == 0) a[q][n] = total;
    }
}

// Ascending bitonic sort of n <= kMaxIncidence 64-bit keys in shared memory.
__device__ void block_sort_u64(unsigned long long* a, int n) {
    const int P = pow2_ceil(max(n, 1));
    for (int i = n + threadIdx.x; i < P; i += blockDim.x) a[i] = ~0ull;
    __syncthreads();
    for (int k = 2; k <= P; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < P; i += blockDim.x) {
                const int l = i ^ j;
                if (l > i) {
                    const unsigned long long x = a[i], y = a[l];
                    if ((x > y) == ((i & k) == 0)) { a[i] = y; a[l] = x; }
                }
            }
            __syncthreads();
        }
}

// Warp-level helpers on global scratch (one warp, all lanes call).
__device__ void warp_sort_int(int* a, int n, int* buf) {
    const int lane = threadIdx.x & 31;
    const int P = pow2_ceil(max(n, 1));
    for (int i = lane; i < P; i += 32) buf[i] = i < n ? a[i] : 0x7fffffff;
    __syncwarp();
    for (int k = 2; k <= P; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = lane; i < P; i += 32) {
                const int l = i ^ j;
                if (l > i) {
                    const int x = buf[i], y = buf[l];
                    if ((x > y) == ((i & k) == 0)) { buf[i] = y; buf[l] = x; }
                }
            }
            __syncwarp();
        }
    for (int i = lane; i < n; i += 32) a[i] = buf[i];
    __syncwarp();
}
__device__ int warp_scan_excl(int* a, int n) {
    const int lane = threadIdx.x & 31;
    int carry = 0;
    for (int base = 0; base < n; base += 32) {
        const int i = base + lane;
        const int v = i < n ? a[i] : 0;
        int x = v;
        for (int o = 1; o < 32; o <<= 1) { const int y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
        if (i < n) a[i] = carry + x - v;
        carry += __shfl_sync(0xffffffffu, x, 31);
    }
    __syncwarp();
    return carry;
}

// ---------------------------------------------------------------------------
// Per-item evaluation
// ---------------------------------------------------------------------------
__device__ __forceinline__ V3 xs3(const double* x, int i) { return ld3(x + i); }
__device__ __forceinline__ int joint_dim(int t) {
    if (t == NXD_JOINT_HINGE || t == NXD_JOINT_FIXED) return 6;
    if (t == NXD_JOINT_PRISMATIC) return 5;
    if (t == NXD_JOINT_CYLINDRICAL) return 4;
    return t == NXD_JOINT_SPHERICAL ? 3 : 2;
}
// inequality joints: value max(C, 0), projected multipliers, active-set Hessian
__device__ __forceinline__ bool joint_is_limit(int t) { return t == NXD_JOINT_ANGLE_LIMIT || t == NXD_JOINT_DISTANCE_LIMIT; }

// JointPrimitives::computeBasis (JointPrimitives.h:29-37) of an axis that the
// joint's constructor has already normalised
__device__ __forceinline__ void joint_basis(V3 axis, V3& u, V3& v) {
    const V3 a = normalized(axis);
    u = fabs(a.x) < 0.8 ? normalized(cross(a, v3(1, 0, 0))) : normalized(cross(a, v3(0, 1, 0)));
    v = normalized(cross(a, u));
}

// Joint residual C at x; with Jd != null also the Jacobian (6 x 12 row-major:
// columns 0-5 body A, 6-11 body B; unused rows zero).  Returns the row count.
__device__ int joint_residual(const Solver& S, int j, const double* x, double* C, double* Jd) {
    const int t = S.jtype[j];
    const int A = S.ja[j], B = S.jb[j];
    const double* P = S.jparams + 16 * j;
    for (int i = 0; i < 6; ++i) C[i] = 0.0;
    if (Jd) for (int e = 0; e < 72; ++e) Jd[e] = 0.0;
    if (t == NXD_JOINT_HINGE || t == NXD_JOINT_SPHERICAL) {
        const V3 pA = xs3(x, 6 * A), pB = xs3(x, 6 * B);
        const Q qA = ldq(S.qj + 4 * A), qB = ldq(S.qj + 4 * B);
        const V3 rA = qrot(qA, ld3(P)), rB = qrot(qB, ld3(P + 3));
        const V3 v = (pA + rA) - (pB + rB);
        C[0] = v.x; C[1] = v.y; C[2] = v.z;
        if (Jd) {
            // PointPrimitive::addJacobianRows (JointPrimitives.h:58-90)
            const M3 dA = cross_mat(rA), dB = cross_mat(rB);
            for (int i = 0; i < 3; ++i) {
                Jd[12 * i + i] = 1.0; Jd[12 * i + 6 + i] = -1.0;
                for (int k = 0; k < 3; ++k) { Jd[12 * i + 3 + k] = -at(dA, i, k); Jd[12 * i + 9 + k] = at(dB, i, k); }
            }
        }
        if (t == NXD_JOINT_SPHERICAL) return 3;
        const V3 nA = qrot(qA, ld3(P + 6)), nB = qrot(qB, ld3(P + 9));
        const V3 c = cross(nA, nB);
        C[3] = c.x; C[4] = c.y; C[5] = c.z;
        if (Jd) {
            // AxisCrossPrimitive::addJacobianRows (JointPrimitives.h:212-240)
            const M3 mA = mat_mul(cross_mat(nB), cross_mat(nA));
            M3 na = cross_mat(nA);
            for (int k = 0; k < 9; ++k) na.m[k] = -na.m[k];
            const M3 mB = mat_mul(na, cross_mat(nB));
            for (int i = 0; i < 3; ++i)
                for (int k = 0; k < 3; ++k) { Jd[12 * (3 + i) + 3 + k] = at(mA, i, k); Jd[12 * (3 + i) + 9 + k] = at(mB, i, k); }
        }
        return 6;
    }
    if (t == NXD_JOINT_FIXED) {
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
        if (Jd) for (int i = 0; i < 6; ++i) Jd[12 * i + i] = 1.0;
        return 6;
    }
    if (t == NXD_JOINT_PRISMATIC || t == NXD_JOINT_CYLINDRICAL) {
        // PrismaticJoint / CylindricalJoint::computeC, computeJ (PrismaticJoint.cpp:30-66,
        // CylindricalJoint.cpp:30-62) from PointOnAxis, Direction and RollLock
        // primitives (JointPrimitives.h:111-265)
        const V3 axA = normalized(ld3(P + 6)), axB = normalized(ld3(P + 9));
        V3 uA, vA, uB, vB;
        joint_basis(axA, uA, vA);
        joint_basis(axB, uB, vB);
        const V3 pA = xs3(x, 6 * A), pB = xs3(x, 6 * B);
        const Q qA = ldq(S.qj + 4 * A), qB = ldq(S.qj + 4 * B);
        const V3 rA = qrot(qA, ld3(P)), rB = qrot(qB, ld3(P + 3));
        const V3 d = (pB + rB) - (pA + rA);
        const V3 uAw = qrot(qA, uA), vAw = qrot(qA, vA);
        C[0] = dot(d, uAw); C[1] = dot(d, vAw);
        const V3 nA = qrot(qA, axA), uBw = qrot(qB, uB), vBw = qrot(qB, vB);
        C[2] = dot(nA, uBw); C[3] = dot(nA, vBw);
        if (Jd) {
            const V3 dirs[2] = {uAw, vAw};
            for (int r = 0; r < 2; ++r) {
                const V3 dir = dirs[r];
                const V3 gA = cross(dir, rA) + cross(dir, d), gB = cross(rB, dir);
                for (int k = 0; k < 3; ++k) {
                    Jd[12 * r + k] = -get(dir, k); Jd[12 * r + 3 + k] = get(gA, k);
                    Jd[12 * r + 6 + k] = get(dir, k); Jd[12 * r + 9 + k] = get(gB, k);
                }
            }
            const V3 bdirs[2] = {uBw, vBw};
            for (int r = 0; r < 2; ++r) {
                const V3 gA = cross(nA, bdirs[r]), gB = cross(bdirs[r], nA);
                for (int k = 0; k < 3; ++k) { Jd[12 * (2 + r) + 3 + k] = get(gA, k); Jd[12 * (2 + r) + 9 + k] = get(gB, k); }
            }
        }
        if (t == NXD_JOINT_CYLINDRICAL) return 4;
        C[4] = dot(uAw, vBw);
        if (Jd) {
            const V3 gA = cross(uAw, vBw), gB = cross(vBw, uAw);
            for (int k = 0; k < 3; ++k) { Jd[12 * 4 + 3 + k] = get(gA, k); Jd[12 * 4 + 9 + k] = get(gB, k); }
        }
        return 5;
    }
    if (t == NXD_JOINT_DISTANCE_LIMIT) {
        // DistanceLimitJoint::computeC / computeJ (DistanceLimitJoint.cpp:38-89)
        const V3 dd = xs3(x, 6 * B) - xs3(x, 6 * A);
        const double dist = norm(dd);
        const V3 dir = dist < 1e-12 ? v3(1, 0, 0) : dd / dist;
        C[0] = P[0] - dist;
        C[1] = dist - dmax(P[1], P[0]);
        if (Jd)
            for (int k = 0; k < 3; ++k) {
                Jd[k] = get(dir, k); Jd[12 + k] = -get(dir, k);
                Jd[6 + k] = -get(dir, k); Jd[12 + 6 + k] = get(dir, k);
            }
        return 2;
    }
    // AngleLimitJoint (AngleLimitJoint.cpp:45-96)
    const Q qA = ldq(S.qj + 4 * A), qB = ldq(S.qj + 4 * B);
    const Q qr = qmul(qconj(qA), qB);
    double ang; V3 ax;
    q_to_angle_axis(qr, ang, ax);
    const V3 axis = ld3(P);
    const double a = ang * dot(ax, axis);
    C[0] = P[3] - a;
    C[1] = a - P[4];
    if (Jd)
        for (int k = 0; k < 3; ++k) {
            Jd[3 + k] = get(axis, k); Jd[12 + 3 + k] = -get(axis, k);
            Jd[9 + k] = -get(axis, k); Jd[12 + 9 + k] = get(axis, k);
        }
    return 2;
}
// Joint::value (Joint.cpp:5-18); AngleLimitJoint::value (AngleLimitJoint.cpp:98-109)
__device__ double joint_energy(const Solver& S, int j, const double* C, int dim) {
    const double mu = S.jmu[j];
    const double* lam = S.jlam + 6 * j;
    if (joint_is_limit(S.jtype[j])) {
        double e = 0.0;
        for (int i = 0; i < 2; ++i) { const double gp = dmax(C[i], 0.0); e += lam[i] * gp + 0.5 * mu * gp * gp; }
        return e;
    }
    double t1 = 0.0, sq = 0.0;
    for (int i = 0; i < dim; ++i) { t1 += lam[i] * C[i]; sq += C[i] * C[i]; }
    return t1 + 0.5 * mu * sq;
}
// C, energy and (full) J and f = mu C + lambda into the per-joint arrays
__device__ void joint_eval(const Solver& S, int j, const double* x, bool full) {
    double C[6];
    const int dim = joint_residual(S, j, x, C, full ? S.jJ + 72 * j : nullptr);
    double* Cj = S.jC + 6 * j;
    for (int i = 0; i < 6; ++i) Cj[i] = C[i];
    S.jE[j] = joint_energy(S, j, C, dim);
    if (!full) return;
    const double mu = S.jmu[j];
    const double* lam = S.jlam + 6 * j;
    double* F = S.jF + 6 * j;
    for (int i = 0; i < 6; ++i) F[i] = 0.0;
    if (joint_is_limit(S.jtype[j])) {
        for (int i = 0; i < 2; ++i) F[i] = C[i] > 0.0 ? lam[i] + mu * C[i] : 0.0;
        S.jact[j] = (C[0] > 0.0 ? 1 : 0) | (C[1] > 0.0 ? 2 : 0);
    } else {
        for (int i = 0; i < dim; ++i) F[i] = mu * C[i] + lam[i];
        S.jact[j] = 0;
    }
}
__device__ __forceinline__ bool joint_couples(const Solver& S, int j) {
    const int t = S.jtype[j];
    if (t == NXD_JOINT_FIXED) return false;
    if (joint_is_limit(t)) return S.jact[j] != 0;
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
__device__ __forceinline__ bool friction_on(const Solver& S, int c) {
    return c < *S.nnf_ptr && S.nforce[c] > 0;
}
// FrictionPotential::value (Friction.cpp:5-20) of contact c at x
__device__ double friction_value(const Solver& S, int c, const double* x) {
    if (!friction_on(S, c)) return 0.0;
    const double N = S.nforce[c];
    const ContactRec& cr = S.contacts[c];
    FricGeom G;
    fric_geom(S, cr, G);
    const V3 u = fric_tangent(S, cr, G, x, *S.dt_ptr);
    const double un = norm(u);
    const double sn = sqrt(un * un + S.friction_eps * S.friction_eps);
    return *S.friction_mu_ptr * N * (sn - S.friction_eps);
}
__device__ void friction_eval(const Solver& S, int c, const double* x, bool full) {
    if (!friction_on(S, c)) { S.fE[c] = 0.0; return; }
    const double N = S.nforce[c];
    const ContactRec& cr = S.contacts[c];
    const double dt = *S.dt_ptr;
    FricGeom G;
    fric_geom(S, cr, G);
    const V3 u = fric_tangent(S, cr, G, x, dt);
    const double mu = *S.friction_mu_ptr, eps = S.friction_eps;
    // FrictionPotential (Friction.cpp:5-61)
    const double un = norm(u);
    const double sn = sqrt(un * un + eps * eps);
    S.fE[c] = mu * N * (sn - eps);
    if (!full) return;
    V3 fg = v3(0, 0, 0);
    double* Hf = S.fHF + 9 * c;
    if (un < 1e-12) {
        const double sc = mu * N / eps;
        for (int i = 0; i < 9; ++i) Hf[i] = (i % 4 == 0) ? sc : 0.0;
    } else {
        const double sc = mu * N / sn;
        fg = sc * u;
        const double s2 = sn * sn;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) Hf[3 * i + j] = sc * ((i == j ? 1.0 : 0.0) - get(u, i) * get(u, j) / s2);
    }
    st3(S.fFG + 3 * c, fg);
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

// Control forms.  VelocityDriveForm (VelocityDriveForm.cpp:61-417) and
// LinearVelocityDriveForm (LinearVelocityDriveForm.cpp:56-280) share the
// stateful joint velocity, on the rotation or the translation part of x;
// PositionDriveForm (PositionDriveForm.cpp:66-172), ForceDriveForm
// (ForceDriveForm.cpp:22-40) and DampedSpringForm (DampedSpringForm.cpp:30-112)
// are stateless.
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
    const int o = S.dkind[d] == NXD_DRIVE_LINEAR_VELOCITY ? 0 : 3;
    const V3 tA = A >= 0 ? xs3(x, 6 * A + o) : v3(0, 0, 0);
    const V3 tB = B >= 0 ? xs3(x, 6 * B + o) : v3(0, 0, 0);
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
// PositionDriveForm::getPositionError
__device__ double position_error(const Solver& S, int d, const double* x) {
    const int A = S.da[d], B = S.db[d];
    const V3 pA = A >= 0 ? xs3(x, 6 * A) : v3(0, 0, 0);
    const V3 pB = B >= 0 ? xs3(x, 6 * B) : v3(0, 0, 0);
    const Drv& p = S.dprm[d];
    return p.vt - dot(pB - pA, v3(p.ax, p.ay, p.az));
}
// DampedSpringForm::springDirection: unit x for a degenerate spring
__device__ V3 spring_direction(const Solver& S, int d, const double* x, double& length) {
    const V3 dv = xs3(x, 6 * S.db[d]) - xs3(x, 6 * S.da[d]);
    length = norm(dv);
    if (length < 1e-12) return v3(1.0, 0.0, 0.0);
    return dv / length;
}
// value of a drive with effective error e and the saturating potential
// (m^2/k) log cosh(k e / m) when the limit m is finite
__device__ double drive_potential(const Drv& p, double e) {
    if (!isfinite(p.maxT)) return 0.5 * p.kv * e * e;
    if (p.kv <= 0.0 || p.maxT <= 0.0) return 0.0;
    const double s = (p.kv * e) / p.maxT;
    return (p.maxT * p.maxT / p.kv) * nxm::log(nxm::cosh(s));
}
// mode 0 value (dE), 1 gradient scalar (dG), 2 Hessian scalar (dH); the
// velocity drives are stateful as in the reference
__device__ void drive_eval(const Solver& S, int d, const double* x, int mode) {
    const Drv& p = S.dprm[d];
    const int kind = S.dkind[d];
    const double dt = *S.dt_ptr;
    if (kind == NXD_DRIVE_FORCE) {
        if (mode == 0) S.dE[d] = 0.0;
        return;
    }
    if (kind == NXD_DRIVE_DAMPED_SPRING) {
        double len;
        const V3 dir = spring_direction(S, d, x, len);
        const double e = len - p.ax;
        if (mode == 0) { S.dE[d] = 0.5 * p.ay * e * e; return; }
        st3(S.dDir + 3 * d, dir);
        if (mode == 1) {
            const double vrel = dot(ld3(S.bvel + 3 * S.db[d]) - ld3(S.bvel + 3 * S.da[d]), dir);
            S.dG[d] = p.ay * e + p.az * vrel;
        } else {
            S.dH[d] = p.ay;
        }
        return;
    }
    if (kind == NXD_DRIVE_POSITION) {
        const double err = position_error(S, d, x);
        if (mode == 0) S.dE[d] = drive_potential(p, drive_dead(p, err));
        else if (mode == 1) S.dG[d] = drive_sat(p, drive_dead(p, err));
        else {
            double h = p.kv;
            if (isfinite(p.maxT) && p.kv > 0.0 && p.maxT > 0.0) {
                if (fabs(err) <= p.delay) h = 0.0;
                else {
                    const double sv = (p.kv * drive_dead(p, err)) / p.maxT;
                    const double th = nxm::tanh(sv);
                    h = p.kv * (1.0 - th * th);
                }
            }
            S.dH[d] = h;
        }
        return;
    }
    const double tgt = drive_target(p, S.dfilt[d]);
    const bool linear = kind == NXD_DRIVE_LINEAR_VELOCITY;
    if (mode == 0) {
        const double v = drive_velocity(S, d, x);
        S.dE[d] = drive_potential(p, drive_dead(p, tgt - v));
    } else if (mode == 1) {
        if (linear) {
            // LinearVelocityDriveForm::gradient: nothing (and no state update) for dt <= 0
            if (dt <= 0) { S.dG[d] = 0.0; return; }
            const double v = drive_velocity(S, d, x);
            S.dG[d] = drive_sat(p, drive_dead(p, tgt - v)) / dt;
            return;
        }
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
                const double sv = (p.kv * ee) / p.maxT;
                const double th = nxm::tanh(sv);
                H = (p.kv * (1.0 - th * th)) / (dt * dt);
            }
        }
        S.dH[d] = H;
    }
}
// Gradient term of drive d at DOF k of its body on `side` (1: body_b): the
// value c the form adds (+1) to or subtracts (-1) from its zeroed gradient,
// or 0 when the form leaves that DOF alone.
__device__ int drive_grad_term(const Solver& S, int d, int side, int k, double& c) {
    const Drv& p = S.dprm[d];
    switch (S.dkind[d]) {
        case NXD_DRIVE_ANGULAR_VELOCITY:
            if (k < 3) return 0;
            c = S.dG[d] * (k == 3 ? p.ax : (k == 4 ? p.ay : p.az));
            return side == 1 ? 1 : -1;
        case NXD_DRIVE_LINEAR_VELOCITY:
        case NXD_DRIVE_POSITION:
            if (k >= 3) return 0;
            c = S.dG[d] * (k == 0 ? p.ax : (k == 1 ? p.ay : p.az));
            return side == 1 ? -1 : 1;
        case NXD_DRIVE_FORCE: {
            const double f[6] = {p.ax, p.ay, p.az, p.kv, p.vt, p.maxT};
            c = f[k];
            return -1;
        }
        default:
            if (k >= 3) return 0;
            c = S.dG[d] * S.dDir[3 * d + k];
            return side == 1 ? 1 : -1;
    }
}
// Translational Hessian entry (h a_r) a_c of a two-body drive (linear and
// position drives: axis; spring: direction), or false when the form emits no
// block (h == 0 for the drives)
__device__ __forceinline__ bool drive_trans_h(const Solver& S, int d, int r, int cc, double& h) {
    const int kind = S.dkind[d];
    if (kind == NXD_DRIVE_DAMPED_SPRING) {
        const double* a = S.dDir + 3 * d;
        h = (S.dH[d] * a[r]) * a[cc];
        return true;
    }
    if (kind != NXD_DRIVE_LINEAR_VELOCITY && kind != NXD_DRIVE_POSITION) return false;
    if (S.dH[d] == 0.0) return false;
    const Drv& p = S.dprm[d];
    const double a[3] = {p.ax, p.ay, p.az};
    h = (S.dH[d] * a[r]) * a[cc];
    return true;
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

// InertiaForm::value (InertiaForm.cpp:14-33) and GravityForm::value
// (GravityForm.cpp:8-16) of body i
__device__ __forceinline__ double inertia_value(const Solver& S, int i, const double* x) {
    const V3 dp = xs3(x, 6 * i) - xs3(S.xhat, 6 * i);
    const double et = 0.5 * S.mass[i] * sqnorm(dp);
    const V3 dth = xs3(x, 6 * i + 3) - xs3(S.xhat, 6 * i + 3);
    const double* I = S.inertia + 9 * i;
    const V3 r = v3(dth.x * I[0] + dth.y * I[3] + dth.z * I[6], dth.x * I[1] + dth.y * I[4] + dth.z * I[7],
                    dth.x * I[2] + dth.y * I[5] + dth.z * I[8]);
    return et + 0.5 * dot(r, dth);
}
__device__ __forceinline__ double gravity_value(const Solver& S, int i, const double* x) {
    return -(S.mass[i] * dot(v3(0.0, -9.81, 0.0), xs3(x, 6 * i)));
}

// ---------------------------------------------------------------------------
// Energies (computeValue / computeContactValue) at x: every per-item term is
// evaluated inside the fixed-tree reduction that sums it (no staging arrays).
// Drives are stateful and evaluated once each before the sums.
// ---------------------------------------------------------------------------
__device__ double energy_total(const Solver& S, const double* x, double s, int C, bool contact_only, BlockRed& R) {
    eval_poses(S, x);
    if (!contact_only)
        for (int d = threadIdx.x; d < S.D; d += blockDim.x) drive_eval(S, d, x, 0);
    __syncthreads();
    const bool bar = *S.barrier_in_forms_ptr != 0, fr = *S.friction_form_ptr != 0;
    const double dh = *S.bdhat_ptr, kap = *S.bkappa_ptr;
    const int n[5] = {contact_only ? 0 : S.N, contact_only ? 0 : S.N, contact_only ? 0 : S.J, bar ? C : 0, fr ? C : 0};
    double sum[5];
    R.sums<5>(n, [&](int q, int e) -> double {
        switch (q) {
            case 0: return inertia_value(S, e, x);
            case 1: return gravity_value(S, e, x);
            case 2: { double Cj[6]; const int dim = joint_residual(S, e, x, Cj, nullptr); return joint_energy(S, e, Cj, dim); }
            case 3: return barrier_value(contact_distance(S.contacts[e], x), dh, kap);
            default: return friction_value(S, e, x);
        }
    }, sum);
    double v = 0.0;
    if (!contact_only) {
        v = sum[0];
        v += s * sum[1];
        v += sum[2];
        for (int d = 0; d < S.D; ++d) v += s * S.dE[d];
        if (S.D > 0) __syncthreads();   // dE is rewritten by the next evaluation
    }
    if (bar) v += s * sum[3];
    if (fr) v += s * sum[4];
    return v;
}

// ---------------------------------------------------------------------------
// Gradient per DOF (item order within each entry), plus the contact-only part
// ---------------------------------------------------------------------------
// inertia, gravity, joints and control forms of DOF (i, k), in that order
__device__ __forceinline__ double gradient_dof_rest(const Solver& S, const double* x, double s, int i, int k) {
    const double m = S.mass[i];
    double g;
    if (k < 3) {
        g = 0.0 + m * (x[6 * i + k] - S.xhat[6 * i + k]);
        const double fgv = k == 1 ? (-m) * -9.81 : (-m) * 0.0;
        g += s * fgv;
    } else {
        const double* I = S.inertia + 9 * i + 3 * (k - 3);
        const double d0 = x[6 * i + 3] - S.xhat[6 * i + 3], d1 = x[6 * i + 4] - S.xhat[6 * i + 4],
                     d2 = x[6 * i + 5] - S.xhat[6 * i + 5];
        g = 0.0 + (I[0] * d0 + I[1] * d1 + I[2] * d2);
        g += s * 0.0;
    }
    // ConstraintForm: J^T (mu C + lambda), joints in order
    double t = 0.0;
    for (int q = S.jinc_off[i]; q < S.jinc_off[i + 1]; ++q) {
        const int j = S.jinc[q] >> 1, side = S.jinc[q] & 1;
        const int dim = joint_dim(S.jtype[j]);
        const double* Jd = S.jJ + 72 * j + 6 * side + k;
        const double* F = S.jF + 6 * j;
        double a = 0.0;
        for (int r = 0; r < dim; ++r) a += Jd[12 * r] * F[r];
        t += a;
    }
    g += t;
    // control forms, each its own form (its zeroed gradient, scaled, added)
    for (int q = S.dinc_off[i]; q < S.dinc_off[i + 1]; ++q) {
        const int d = S.dinc[q] >> 1, side = S.dinc[q] & 1;
        double c = 0.0;
        const int sg = drive_grad_term(S, d, side, k, c);
        const double tk = sg == 0 ? 0.0 : (sg > 0 ? 0.0 + c : 0.0 - c);
        g += s * tk;
    }
    return g;
}
// contact terms of DOF (i, k) for contact end q: barrier (bit 1) and friction (bit 2)
__device__ __forceinline__ int gradient_contact_terms(const Solver& S, int q, int k, bool bar, bool fr, double dh,
                                                      double& tb, double& tf) {
    const int c = S.cinc[q] >> 1, side = S.cinc[q] & 1;
    int fl = 0;
    tb = 0.0; tf = 0.0;
    if (bar && k < 3 && S.bD[c] < dh) {
        const double gpv = S.bGP[c];
        const double nk = S.contacts[c].normal[k];
        tb = side == 0 ? (-gpv) * nk : gpv * nk;
        fl |= 1;
    }
    if (fr && friction_on(S, c)) {
        const double* Jx = (side == 0 ? S.fJA : S.fJB) + 18 * c;
        const double* fg = S.fFG + 3 * c;
        tf = Jx[k] * fg[0] + Jx[6 + k] * fg[1] + Jx[12 + k] * fg[2];
        fl |= 2;
    }
    return fl;
}
__device__ __forceinline__ void gradient_dof_finish(double g, double cb, double cf, double s, bool bar, bool fr,
                                                    double& g_out, double& cg_out) {
    double cgv = 0.0;
    if (bar) { g += s * cb; cgv += s * cb; }
    if (fr) { g += s * cf; cgv += s * cf; }
    g_out = g;
    cg_out = cgv;
}
__device__ void gradient_dof(const Solver& S, const double* x, double s, int i, int k, bool bar, bool fr, double dh,
                             double& g_out, double& cg_out) {
    const double g = gradient_dof_rest(S, x, s, i, k);
    double cb = 0.0, cf = 0.0;
    if (bar || fr) {
        for (int q = S.cinc_off[i]; q < S.cinc_off[i + 1]; ++q) {
            const int c = S.cinc[q] >> 1, side = S.cinc[q] & 1;
            if (bar && k < 3 && S.bD[c] < dh) {
                const double gpv = S.bGP[c];
                const double nk = S.contacts[c].normal[k];
                cb += side == 0 ? (-gpv) * nk : gpv * nk;
            }
            if (fr && friction_on(S, c)) {
                const double* Jx = (side == 0 ? S.fJA : S.fJB) + 18 * c;
                const double* fg = S.fFG + 3 * c;
                cf += Jx[k] * fg[0] + Jx[6 + k] * fg[1] + Jx[12 + k] * fg[2];
            }
        }
    }
    gradient_dof_finish(g, cb, cf, s, bar, fr, g_out, cg_out);
}
// gradient_dof by one warp (every lane returns the same values): each lane
// evaluates one contact end's terms per round, tw (256 doubles of shared
// memory per warp) holds a round's terms, and every lane adds them in
// contact order, so each sum is the same double as the sequential loop's.
__device__ void gradient_dof_warp(const Solver& S, const double* x, double s, int i, int k, bool bar, bool fr,
                                  double dh, double& g_out, double& cg_out, double* tw) {
    const int lane = threadIdx.x & 31;
    const double g = gradient_dof_rest(S, x, s, i, k);
    double cb = 0.0, cf = 0.0;
    if (bar || fr) {
        const int q0 = S.cinc_off[i], q1 = S.cinc_off[i + 1];
        int* fw = reinterpret_cast<int*>(tw + 64);
        for (int base = q0; base < q1; base += 32) {
            double tb = 0.0, tf = 0.0;
            int fl = 0;
            if (base + lane < q1) fl = gradient_contact_terms(S, base + lane, k, bar, fr, dh, tb, tf);
            tw[lane] = tb;
            tw[32 + lane] = tf;
            fw[lane] = fl;
            __syncwarp();
            const int cnt = min(32, q1 - base);
            for (int j = 0; j < cnt; ++j) {
                const int f = fw[j];
                if (f & 1) cb += tw[j];
                if (f & 2) cf += tw[32 + j];
            }
            __syncwarp();
        }
    }
    gradient_dof_finish(g, cb, cf, s, bar, fr, g_out, cg_out);
}
__device__ void gather_gradient(const Solver& S, const double* x, double s, int C) {
    const bool bar = *S.barrier_in_forms_ptr != 0, fr = *S.friction_form_ptr != 0;
    const double dh = *S.bdhat_ptr;
    for (int e = threadIdx.x; e < 6 * S.N; e += blockDim.x) {
        double g, cg;
        gradient_dof(S, x, s, e / 6, e % 6, bar, fr, dh, g, cg);
        S.g[e] = g;
        S.cg[e] = cg;
    }
}

// ---------------------------------------------------------------------------
// Hessian: diagonal block per body (one thread per block row), coupling
// blocks per item
// ---------------------------------------------------------------------------
// row a of the 6x6 block mu J_ra^T J_ca of a base joint
__device__ __forceinline__ void joint_block_row(const Solver& S, int j, int ra, int ca, int a, double* out) {
    const int dim = joint_dim(S.jtype[j]);
    const double* Jd = S.jJ + 72 * j;
    const double mu = S.jmu[j];
    for (int b = 0; b < 6; ++b) {
        double sacc = 0.0;
        for (int r = 0; r < dim; ++r) sacc += Jd[12 * r + 6 * ra + a] * Jd[12 * r + 6 * ca + b];
        out[b] = sacc * mu;
    }
}
__device__ void joint_block(const Solver& S, int j, int ra, int ca, double* out) {
    for (int a = 0; a < 6; ++a) joint_block_row(S, j, ra, ca, a, out + 6 * a);
}
// entry (a, b) of the 3x3 rotational AngleLimit block sum_active mu axis axis^T
__device__ __forceinline__ double angle_limit_h(const Solver& S, int j, int a, int b) {
    const double* ax = S.jparams + 16 * j;
    const double mu = S.jmu[j];
    double h = 0.0;
    for (int rep = 0; rep < 2; ++rep)
        if (S.jact[j] & (1 << rep)) h += mu * (ax[a] * ax[b]);
    return h;
}
// entry (a, b) of the translational DistanceLimit block sum_active mu dir dir^T
// (DistanceLimitJoint.cpp:113-160); dir is row 0 of the stored Jacobian
__device__ __forceinline__ double distance_limit_h(const Solver& S, int j, int a, int b) {
    const double* dir = S.jJ + 72 * j;
    const double mu = S.jmu[j];
    double h = 0.0;
    for (int rep = 0; rep < 2; ++rep)
        if (S.jact[j] & (1 << rep)) h += mu * (dir[a] * dir[b]);
    return h;
}
__device__ void angle_limit_H(const Solver& S, int j, double* H3) {
    for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) H3[3 * a + b] = angle_limit_h(S, j, a, b);
}
// row r of the friction block J_X^T Hf J_Y, evaluated (J_X^T Hf) J_Y
__device__ __forceinline__ void friction_block_row(const Solver& S, int c, int sx, int sy, int r, double* out) {
    const double* Jx = (sx == 0 ? S.fJA : S.fJB) + 18 * c;
    const double* Jy = (sy == 0 ? S.fJA : S.fJB) + 18 * c;
    const double* Hf = S.fHF + 9 * c;
    const double T0 = Jx[r] * Hf[0] + Jx[6 + r] * Hf[3] + Jx[12 + r] * Hf[6];
    const double T1 = Jx[r] * Hf[1] + Jx[6 + r] * Hf[4] + Jx[12 + r] * Hf[7];
    const double T2 = Jx[r] * Hf[2] + Jx[6 + r] * Hf[5] + Jx[12 + r] * Hf[8];
    for (int cc = 0; cc < 6; ++cc) out[cc] = T0 * Jy[cc] + T1 * Jy[6 + cc] + T2 * Jy[12 + cc];
}
__device__ void friction_block(const Solver& S, int c, int sx, int sy, double* out) {
    for (int r = 0; r < 6; ++r) friction_block_row(S, c, sx, sy, r, out + 6 * r);
}
// drive Hessian entry (ra, ca) of the rotational block (upper entries use
// (H a_r) a_c with r <= c, the mirrored lower ones repeat them)
__device__ __forceinline__ double drive_h(const Solver& S, int d, int ra, int ca, double s) {
    const Drv& p = S.dprm[d];
    const double ax[3] = {p.ax, p.ay, p.az};
    const double Hd = S.dH[d];
    const int lo = min(ra, ca), hi = max(ra, ca);
    return (Hd * ax[lo] * ax[hi]) * s;
}

// row a of body i's diagonal block: inertia, joints and control forms
__device__ __forceinline__ void diag_hessian_row_rest(const Solver& S, double s, int i, int a, double* H) {
    for (int b = 0; b < 6; ++b) H[b] = 0.0;
    if (a < 3) H[a] += S.mass[i];
    else for (int b = 0; b < 3; ++b) H[3 + b] += S.inertia[9 * i + 3 * (a - 3) + b];
    double blk[6];
    for (int q = S.jinc_off[i]; q < S.jinc_off[i + 1]; ++q) {
        const int j = S.jinc[q] >> 1, side = S.jinc[q] & 1;
        if (S.jtype[j] == NXD_JOINT_ANGLE_LIMIT) {
            if (!S.jact[j]) continue;
            if (a >= 3) for (int b = 0; b < 3; ++b) H[3 + b] += angle_limit_h(S, j, a - 3, b);
        } else if (S.jtype[j] == NXD_JOINT_DISTANCE_LIMIT) {
            if (!S.jact[j]) continue;
            if (a < 3) for (int b = 0; b < 3; ++b) H[b] += distance_limit_h(S, j, a, b);
        } else {
            joint_block_row(S, j, side, side, a, blk);
            for (int b = 0; b < 6; ++b) H[b] += blk[b];
        }
    }
    for (int q = S.dinc_off[i]; q < S.dinc_off[i + 1]; ++q) {
        const int d = S.dinc[q] >> 1;
        if (S.dkind[d] == NXD_DRIVE_ANGULAR_VELOCITY) {
            if (S.dH[d] == 0.0) continue;
            if (a >= 3) for (int b = 0; b < 3; ++b) H[3 + b] += drive_h(S, d, a - 3, b, s);
        } else if (a < 3) {
            double h;
            for (int b = 0; b < 3; ++b)
                if (drive_trans_h(S, d, a, b, h)) H[b] += h * s;
        }
    }
}
// row a of body i's diagonal block, contributions in item order
__device__ void diag_hessian_row(const Solver& S, double s, int i, int a, bool bar, bool fr, double dh, double* H) {
    double blk[6];
    diag_hessian_row_rest(S, s, i, a, H);
    if (!(bar || fr)) return;
    if (bar && a < 3)
        for (int q = S.cinc_off[i]; q < S.cinc_off[i + 1]; ++q) {
            const int c = S.cinc[q] >> 1;
            if (!(S.bD[c] < dh)) continue;
            const double hp = S.bHP[c];
            const double* n = S.contacts[c].normal;
            for (int cc = 0; cc < 3; ++cc) H[cc] += (hp * (n[a] * n[cc])) * s;
        }
    if (fr)
        for (int q = S.cinc_off[i]; q < S.cinc_off[i + 1]; ++q) {
            const int c = S.cinc[q] >> 1, side = S.cinc[q] & 1;
            if (!friction_on(S, c)) continue;
            friction_block_row(S, c, side, side, a, blk);
            for (int b = 0; b < 6; ++b) H[b] += blk[b] * s;
        }
}
// diag_hessian_row by one warp (every lane returns the same row): the
// barrier pass, then the friction pass, each a round of 32 contact ends whose
// terms the lanes evaluate and every lane adds in contact order (tw: 256
// doubles of shared memory per warp).
__device__ void diag_hessian_row_warp(const Solver& S, double s, int i, int a, bool bar, bool fr, double dh, double* H,
                                      double* tw) {
    const int lane = threadIdx.x & 31;
    diag_hessian_row_rest(S, s, i, a, H);
    if (!(bar || fr)) return;
    const int q0 = S.cinc_off[i], q1 = S.cinc_off[i + 1];
    int* fw = reinterpret_cast<int*>(tw + 192);
    for (int pass = 0; pass < 2; ++pass) {
        if (pass == 0 && !(bar && a < 3)) continue;
        if (pass == 1 && !fr) continue;
        for (int base = q0; base < q1; base += 32) {
            const int q = base + lane;
            int fl = 0;
            double v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
            if (q < q1) {
                const int c = S.cinc[q] >> 1, side = S.cinc[q] & 1;
                if (pass == 0) {
                    if (S.bD[c] < dh) {
                        const double hp = S.bHP[c];
                        const double* n = S.contacts[c].normal;
                        for (int cc = 0; cc < 3; ++cc) v[cc] = (hp * (n[a] * n[cc])) * s;
                        fl = 1;
                    }
                } else if (friction_on(S, c)) {
                    double blk[6];
                    friction_block_row(S, c, side, side, a, blk);
                    for (int b = 0; b < 6; ++b) v[b] = blk[b] * s;
                    fl = 1;
                }
            }
            for (int b = 0; b < 6; ++b) tw[32 * b + lane] = v[b];
            fw[lane] = fl;
            __syncwarp();
            const int cnt = min(32, q1 - base), nb = pass == 0 ? 3 : 6;
            for (int j = 0; j < cnt; ++j) {
                if (!fw[j]) continue;
                for (int b = 0; b < nb; ++b) H[b] += tw[32 * b + j];
            }
            __syncwarp();
        }
    }
}
__device__ void gather_diag_hessian(const Solver& S, double s, int C) {
    const bool bar = *S.barrier_in_forms_ptr != 0, fr = *S.friction_form_ptr != 0;
    const double dh = *S.bdhat_ptr;
    for (int e = threadIdx.x; e < 6 * S.N; e += blockDim.x) {
        double H[6];
        diag_hessian_row(S, s, e / 6, e % 6, bar, fr, dh, H);
        for (int b = 0; b < 6; ++b) S.Hd[6 * e + b] = H[b];
    }
}

// Coupling block entry e (row-major 6x6) of item `it` with rows of body R
// and cols of body Cb (R != Cb).  Items, in the order their triplets reach
// the Hessian: [0,J) joints, [J,J+D) control forms, [J+D, J+D+C) barrier
// contacts, [J+D+C, J+D+2C) friction contacts.
__device__ double coupling_entry(const Solver& S, int it, int R, int Cb, double s, int C, int e) {
    if (S.ext_n >= 0) return S.ext_row[it] == R ? S.ext_vals[36LL * it + e] : 0.0;   // block (R, Cb) as stored
    const int ra = e / 6, cb = e % 6;
    if (it >= S.J && it < S.J + S.D) {
        // two-body control form: -(h a_ra) a_cb in both off-diagonal blocks
        double h;
        if (ra >= 3 || cb >= 3 || !drive_trans_h(S, it - S.J, ra, cb, h)) return 0.0;
        return (-h) * s;
    }
    if (it < S.J) {
        const int j = it;
        if (S.jtype[j] == NXD_JOINT_ANGLE_LIMIT)
            return (ra >= 3 && cb >= 3) ? -angle_limit_h(S, j, ra - 3, cb - 3) : 0.0;
        if (S.jtype[j] == NXD_JOINT_DISTANCE_LIMIT)
            return (ra < 3 && cb < 3) ? -distance_limit_h(S, j, ra, cb) : 0.0;
        const int sr = S.ja[j] == R ? 0 : 1, sc = S.ja[j] == Cb ? 0 : 1;
        const int dim = joint_dim(S.jtype[j]);
        const double* Jd = S.jJ + 72 * j;
        double acc = 0.0;
        for (int r = 0; r < dim; ++r) acc += Jd[12 * r + 6 * sr + ra] * Jd[12 * r + 6 * sc + cb];
        return acc * S.jmu[j];
    }
    const int J2 = S.J + S.D;
    if (it < J2 + C) {
        if (ra >= 3 || cb >= 3) return 0.0;
        const int c = it - J2;
        const double* n = S.contacts[c].normal;
        return (-(S.bHP[c] * (n[ra] * n[cb]))) * s;
    }
    const int c = it - J2 - C;
    const int sx = S.contacts[c].body_a == R ? 0 : 1, sy = S.contacts[c].body_a == Cb ? 0 : 1;
    const double* Jx = (sx == 0 ? S.fJA : S.fJB) + 18 * c;
    const double* Jy = (sy == 0 ? S.fJA : S.fJB) + 18 * c;
    const double* Hf = S.fHF + 9 * c;
    const double T0 = Jx[ra] * Hf[0] + Jx[6 + ra] * Hf[3] + Jx[12 + ra] * Hf[6];
    const double T1 = Jx[ra] * Hf[1] + Jx[6 + ra] * Hf[4] + Jx[12 + ra] * Hf[7];
    const double T2 = Jx[ra] * Hf[2] + Jx[6 + ra] * Hf[5] + Jx[12 + ra] * Hf[8];
    return (T0 * Jy[cb] + T1 * Jy[6 + cb] + T2 * Jy[12 + cb]) * s;
}
// whole block, added into out (used by the form interface)
__device__ void add_coupling_block(const Solver& S, int it, int R, int Cb, double s, double* out) {
    const int C = *S.ncontacts_ptr;
    for (int e = 0; e < 36; ++e) {
        const int ra = e / 6, cb = e % 6;
        const bool touches = it < S.J ? (S.jtype[it] == NXD_JOINT_ANGLE_LIMIT ? (ra >= 3 && cb >= 3)
                                         : (S.jtype[it] == NXD_JOINT_DISTANCE_LIMIT ? (ra < 3 && cb < 3) : true))
                                      : (it < S.J + S.D + C ? (ra < 3 && cb < 3) : true);
        if (touches) out[e] += coupling_entry(S, it, R, Cb, s, C, e);
    }
}
__device__ __forceinline__ void item_bodies(const Solver& S, int it, int& a, int& b) {
    if (S.ext_n >= 0) { a = S.ext_row[it]; b = S.ext_col[it]; return; }
    if (it < S.J) { a = S.ja[it]; b = S.jb[it]; return; }
    const int J2 = S.J + S.D;
    if (it < J2) { a = S.da[it - S.J]; b = S.db[it - S.J]; return; }
    const int C = *S.ncontacts_ptr;
    const int c = it < J2 + C ? it - J2 : it - J2 - C;
    a = S.contacts[c].body_a; b = S.contacts[c].body_b;
}
// a control form couples its two bodies when it emits off-diagonal blocks:
// the spring always, the linear and position drives when h != 0
__device__ __forceinline__ bool drive_couples(const Solver& S, int d) {
    if (S.da[d] < 0) return false;
    const int kind = S.dkind[d];
    if (kind == NXD_DRIVE_DAMPED_SPRING) return true;
    return (kind == NXD_DRIVE_LINEAR_VELOCITY || kind == NXD_DRIVE_POSITION) && S.dH[d] != 0.0;
}
__device__ __forceinline__ bool item_active(const Solver& S, int it) {
    if (S.ext_n >= 0) return S.ext_row[it] != S.ext_col[it];
    if (it < S.J) return joint_couples(S, it);
    const int J2 = S.J + S.D;
    if (it < J2) return drive_couples(S, it - S.J);
    const int C = *S.ncontacts_ptr;
    if (it < J2 + C) return *S.barrier_in_forms_ptr != 0 && S.bD[it - J2] < *S.bdhat_ptr;
    const int c = it - J2 - C;
    return *S.friction_form_ptr != 0 && friction_on(S, c);
}

// ---------------------------------------------------------------------------
// Contact incidence: body -> (contact * 2 + side), ascending, from one sort of
// (body, end) keys; cinc_off[b] = first key of body >= b.
// ---------------------------------------------------------------------------
__device__ void build_contact_incidence(const Solver& S, int C, unsigned long long* keys) {
    const int n = 2 * C;
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
        const ContactRec& cr = S.contacts[e >> 1];
        const int b = (e & 1) ? cr.body_b : cr.body_a;
        keys[e] = ((unsigned long long)(unsigned)b << 32) | (unsigned)e;
    }
    block_sort_u64(keys, n);
    for (int p = threadIdx.x; p <= n; p += blockDim.x) {
        const int lo = p == 0 ? -1 : (int)(keys[p - 1] >> 32);
        const int hi = p == n ? S.N : (int)(keys[p] >> 32);
        for (int b = lo + 1; b <= hi; ++b) S.cinc_off[b] = p;
        if (p < n) S.cinc[p] = (int)(keys[p] & 0xffffffffu);
    }
    __syncthreads();
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

// LDL^T of one 6x6 block (lower part of H), left-looking exactly as the dense
// oracle loop, solving rhs in place.  Fully unrolled: A stays in registers.
// Returns false on a zero pivot.
__device__ __forceinline__ bool ldlt6_solve(double (&A)[36], double (&b)[6]) {
    double d[6];
#pragma unroll
    for (int j = 0; j < 6; ++j) {
        double dj = A[6 * j + j];
#pragma unroll
        for (int k = 0; k < j; ++k) { const double l = A[6 * j + k]; dj -= l * l * d[k]; }
        if (dj == 0.0) return false;
        d[j] = dj;
        A[6 * j + j] = dj;
#pragma unroll
        for (int i = j + 1; i < 6; ++i) {
            double s = A[6 * i + j];
#pragma unroll
            for (int k = 0; k < j; ++k) s -= A[6 * i + k] * A[6 * j + k] * d[k];
            A[6 * i + j] = s / dj;
        }
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        double s = b[i];
#pragma unroll
        for (int k = 0; k < i; ++k) s -= A[6 * i + k] * b[k];
        b[i] = s;
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) b[i] /= A[6 * i + i];
#pragma unroll
    for (int i = 5; i >= 0; --i) {
        double s = b[i];
#pragma unroll
        for (int k = 5; k > i; --k) s -= A[6 * k + i] * b[k];
        b[i] = s;
    }
    return true;
}

// ---------------------------------------------------------------------------
// Block-sparse LDL^T of one multi-body component, one warp.
//
// Members are put in elimination order by (distinct coupled neighbours, body
// index).  The block structure of L (with fill) comes from bit masks:
// colm[p] = rows below p, filled by merging each column into its parent (the
// first row below it); rowm[i] = the columns of row i.  L is stored by block
// rows (row i's blocks in ascending column order), D with the strictly lower
// part of each diagonal block.  Column p is computed left-looking: every entry
// first takes the updates (L_ik L_pk) d_k of all earlier structurally nonzero
// block columns k in ascending order, then those of the columns of block p
// before it, in registers (one lane per row of the panel, 30 rows per pass).
// Forward substitution is fused into the column loop; backward substitution
// runs in descending block order.  Every entry sees the same sequence of
// operations as the dense oracle loop (its skipped terms are exact zeros).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int mask_rank(const unsigned* row, int b) {
    int r = 0;
    for (int w = 0; w < (b >> 5); ++w) r += __popc(row[w]);
    return r + __popc(row[b >> 5] & ((1u << (b & 31)) - 1u));
}
__device__ __forceinline__ bool mask_test(const unsigned* row, int b) { return (row[b >> 5] >> (b & 31)) & 1u; }

// returns 0 ok, 1 zero pivot, 2 capacity
// Workspace: the structure words, then the factor doubles, each in the warp's
// shared-memory slab when it fits there, else in the global pools.  With
// reuse, the slab already holds this component's structure (same members,
// items and coupling pattern): only the numeric part runs.  in_slab tells
// the caller whether the structure now sits in the slab.
__device__ int solve_component(const Solver& S, int root, double s, int C, unsigned char* slab, bool reuse,
                               bool& in_slab) {
    const int lane = threadIdx.x & 31;
    const unsigned full = 0xffffffffu;
    const int k = S.mcnt[root + 1] - S.mcnt[root];
    const int m = S.icnt[root + 1] - S.icnt[root];
    int* mem = S.members + S.mcnt[root];
    int* its = S.items + S.icnt[root];
    if (k > kMaxComponentBodies) return 2;
    const int W = (k + 31) >> 5;
    const int Psort = max(pow2_ceil(k), pow2_ceil(max(m, 1)));
    const long long nwords = Psort + 3LL * k * W + 6LL * k + 2;
    unsigned* base;
    size_t slab_used = 0;
    in_slab = false;
    if (slab && 4 * nwords <= S.slab_bytes) {
        base = reinterpret_cast<unsigned*>(slab);
        slab_used = (size_t)(4 * nwords + 15) & ~(size_t)15;
        in_slab = true;
    } else {
        reuse = false;
        long long off = 0;
        if (lane == 0) off = (long long)atomicAdd((unsigned long long*)S.mpool_off, (unsigned long long)nwords);
        off = __shfl_sync(full, off, 0);
        if (off + nwords > S.mpool_cap) return 2;
        base = S.mpool + off;
    }
    int* sortbuf = (int*)base;
    unsigned* adj = base + Psort;
    unsigned* colm = adj + (size_t)k * W;
    unsigned* rowm = colm + (size_t)k * W;
    int* deg = (int*)(rowm + (size_t)k * W);
    int* degcnt = deg + k;
    int* pos_of = degcnt + k + 1;
    int* body_at = pos_of + k;
    int* rowptr = body_at + k;
    int* rows = rowptr + k + 1;
    const unsigned lt = (1u << lane) - 1u;
    int nnz;
    if (reuse) {
        nnz = rowptr[k];
    } else {
    // members ascending, items in item order
    warp_sort_int(mem, k, sortbuf);
    warp_sort_int(its, m, sortbuf);
    for (int t = lane; t < k; t += 32) S.local[mem[t]] = t;
    for (long long e = lane; e < 3LL * k * W; e += 32) adj[e] = 0u;
    for (int t = lane; t <= k; t += 32) degcnt[t] = 0;
    __syncwarp();
    for (int q = lane; q < m; q += 32) {
        int a, b;
        item_bodies(S, its[q], a, b);
        const int la = S.local[a], lb = S.local[b];
        atomicOr(&adj[la * W + (lb >> 5)], 1u << (lb & 31));
        atomicOr(&adj[lb * W + (la >> 5)], 1u << (la & 31));
    }
    __syncwarp();
    for (int t = lane; t < k; t += 32) {
        int d = 0;
        for (int w = 0; w < W; ++w) d += __popc(adj[t * W + w]);
        deg[t] = d;
        atomicAdd(&degcnt[d], 1);
    }
    __syncwarp();
    warp_scan_excl(degcnt, k + 1);
    // stable counting placement by degree (members already ascending)
    for (int b0 = 0; b0 < k; b0 += 32) {
        const int t = b0 + lane;
        const int key = t < k ? deg[t] : -1 - lane;
        const unsigned mask = __match_any_sync(full, key);
        const int rank = __popc(mask & lt);
        const int start = t < k ? degcnt[key] : 0;
        __syncwarp();
        if (t < k) { pos_of[t] = start + rank; body_at[start + rank] = mem[t]; }
        if (t < k && lane == __ffs(mask) - 1) degcnt[key] = start + __popc(mask);
        __syncwarp();
    }
    // lower structure in elimination positions
    for (int t = lane; t < k; t += 32) {
        const int pt = pos_of[t];
        for (int w = 0; w < W; ++w) {
            unsigned mm = adj[t * W + w];
            while (mm) {
                const int u = 32 * w + __ffs(mm) - 1;
                mm &= mm - 1;
                const int pu = pos_of[u];
                if (pu > pt) atomicOr(&colm[pt * W + (pu >> 5)], 1u << (pu & 31));
            }
        }
    }
    __syncwarp();
    // symbolic fill: column p merges into its parent
    for (int p = 0; p < k; ++p) {
        const unsigned w0 = lane < W ? colm[p * W + lane] : 0u;
        const unsigned w1 = lane + 32 < W ? colm[p * W + lane + 32] : 0u;
        const unsigned b0 = __ballot_sync(full, w0 != 0u), b1 = __ballot_sync(full, w1 != 0u);
        if (!b0 && !b1) continue;
        int wi;
        unsigned word;
        if (b0) { wi = __ffs(b0) - 1; word = __shfl_sync(full, w0, wi); }
        else { const int l1 = __ffs(b1) - 1; word = __shfl_sync(full, w1, l1); wi = 32 + l1; }
        const int par = 32 * wi + __ffs(word) - 1;
        unsigned v0 = w0, v1 = w1;
        if (lane == wi) v0 &= ~(1u << (par & 31));
        if (lane + 32 == wi) v1 &= ~(1u << (par & 31));
        if (v0) colm[par * W + lane] |= v0;
        if (v1) colm[par * W + lane + 32] |= v1;
        __syncwarp();
    }
    for (int p = lane; p < k; p += 32)
        for (int w = 0; w < W; ++w) {
            unsigned mm = colm[p * W + w];
            while (mm) {
                const int i = 32 * w + __ffs(mm) - 1;
                mm &= mm - 1;
                atomicOr(&rowm[i * W + (p >> 5)], 1u << (p & 31));
            }
        }
    __syncwarp();
    for (int i = lane; i < k; i += 32) {
        int c = 0;
        for (int w = 0; w < W; ++w) c += __popc(rowm[i * W + w]);
        rowptr[i] = c;
    }
    __syncwarp();
    nnz = warp_scan_excl(rowptr, k);
    if (lane == 0) rowptr[k] = nnz;
    }
    const long long ndoubles = 36LL * (k + nnz) + 6LL * k;
    double* Dg;
    if (slab && (long long)slab_used + 8 * ndoubles <= S.slab_bytes) {
        Dg = reinterpret_cast<double*>(slab + slab_used);
    } else {
        long long doff = 0;
        if (lane == 0) doff = (long long)atomicAdd((unsigned long long*)S.pool_off, (unsigned long long)ndoubles);
        doff = __shfl_sync(full, doff, 0);
        if (doff + ndoubles > S.pool_cap) return 2;
        Dg = S.pool + doff;
    }
    double* Lv = Dg + 36LL * k;
    double* vec = Lv + 36LL * nnz;
    for (int e = lane; e < 36 * k; e += 32) Dg[e] = S.Hd[36 * body_at[e / 36] + e % 36];
    for (long long e = lane; e < 36LL * nnz; e += 32) Lv[e] = 0.0;
    for (int e = lane; e < 6 * k; e += 32) vec[e] = -S.g[6 * body_at[e / 6] + e % 6];
    __syncwarp();
    // coupling blocks, items in item order (lane e owns entry e of every block)
    for (int q = 0; q < m; ++q) {
        const int it = its[q];
        int a, b;
        item_bodies(S, it, a, b);
        const int pa = pos_of[S.local[a]], pb = pos_of[S.local[b]];
        const int R = pa > pb ? a : b, Cb = pa > pb ? b : a;
        const int I = max(pa, pb), Jc = min(pa, pb);
        double* blk = Lv + 36LL * (rowptr[I] + mask_rank(rowm + (size_t)I * W, Jc));
        for (int e = lane; e < 36; e += 32) blk[e] += coupling_entry(S, it, R, Cb, s, C, e);
    }
    __syncwarp();

    // numeric factorisation with fused forward substitution
    for (int p = 0; p < k; ++p) {
        const unsigned* rp = rowm + (size_t)p * W;
        // rows of column p, ascending
        int nb = 0;
        for (int b0 = ((p + 1) >> 5) << 5; b0 < k; b0 += 32) {
            const int bit = b0 + lane;
            const bool set = bit > p && bit < k && mask_test(colm + (size_t)p * W, bit);
            const unsigned bal = __ballot_sync(full, set);
            if (set) rows[nb + __popc(bal & lt)] = bit;
            nb += __popc(bal);
        }
        __syncwarp();
        double Lr[6], dJ[6];
        for (int chunk = 0;; ++chunk) {
            const bool diag = chunk == 0 && lane < 6;
            const int bi = chunk == 0 ? (lane - 6) / 6 : 4 + 5 * (chunk - 1) + lane / 6;
            const int r = diag ? lane : (chunk == 0 ? (lane - 6) % 6 : lane % 6);
            const bool valid = diag || (lane < 30 && (chunk > 0 || lane >= 6) && bi < nb);
            const int I = diag || !valid ? p : rows[bi];
            double T[6];
            double* Lrow = nullptr;
            for (int c = 0; c < 6; ++c) Lr[c] = 0.0;
            if (valid) {
                if (diag) {
                    for (int c = 0; c < 6; ++c) T[c] = Dg[36LL * p + 6 * r + c];
                } else {
                    Lrow = Lv + 36LL * (rowptr[I] + mask_rank(rowm + (size_t)I * W, p)) + 6 * r;
                    for (int c = 0; c < 6; ++c) T[c] = Lrow[c];
                }
                // updates of the earlier block columns K in rowm[I] & rowm[p]
                const unsigned* ri = rowm + (size_t)I * W;
                int cI = 0, cP = 0;
                for (int w = 0; w < W; ++w) {
                    const unsigned mi = ri[w], mp = rp[w];
                    unsigned both = mi & mp;
                    while (both) {
                        const int bb = __ffs(both) - 1;
                        both &= both - 1;
                        const unsigned below = (1u << bb) - 1u;
                        const double* Lik = Lv + 36LL * (rowptr[I] + cI + __popc(mi & below)) + 6 * r;
                        const double* Lpk = Lv + 36LL * (rowptr[p] + cP + __popc(mp & below));
                        const double* dK = Dg + 36LL * (32 * w + bb);
                        for (int kk = 0; kk < 6; ++kk) {
                            const double lik = Lik[kk], dk = dK[7 * kk];
                            for (int c = 0; c < 6; ++c) T[c] -= (lik * Lpk[6 * c + kk]) * dk;
                        }
                    }
                    cI += __popc(mi);
                    cP += __popc(mp);
                }
            } else {
                for (int c = 0; c < 6; ++c) T[c] = 0.0;
            }
            // the six columns of block p
            for (int c = 0; c < 6; ++c) {
                double val = T[c];
                if (chunk == 0) {
                    for (int c2 = 0; c2 < c; ++c2) {
                        const double lcc = __shfl_sync(full, Lr[c2], c);
                        val -= (Lr[c2] * lcc) * dJ[c2];
                    }
                    dJ[c] = __shfl_sync(full, val, c);
                } else {
                    for (int c2 = 0; c2 < c; ++c2) val -= (Lr[c2] * Dg[36LL * p + 6 * c + c2]) * dJ[c2];
                }
                if (dJ[c] == 0.0) return 1;
                if (valid && !(diag && r <= c)) Lr[c] = val / dJ[c];
            }
            if (valid) {
                if (diag) {
                    for (int c = 0; c < r; ++c) Dg[36LL * p + 6 * r + c] = Lr[c];
                    Dg[36LL * p + 7 * r] = dJ[r];
                } else {
                    for (int c = 0; c < 6; ++c) Lrow[c] = Lr[c];
                }
            }
            __syncwarp();
            if (chunk == 0) {
                // forward substitution for block p (lanes 0-5 hold its rows)
                double yv = 0.0;
                if (lane < 6) {
                    yv = vec[6 * p + lane];
                    int cP = 0;
                    for (int w = 0; w < W; ++w) {
                        const unsigned mp = rp[w];
                        unsigned mm = mp;
                        while (mm) {
                            const int bb = __ffs(mm) - 1;
                            mm &= mm - 1;
                            const double* Lpk = Lv + 36LL * (rowptr[p] + cP + __popc(mp & ((1u << bb) - 1u))) + 6 * lane;
                            const double* yk = vec + 6 * (32 * w + bb);
                            for (int kk = 0; kk < 6; ++kk) yv -= Lpk[kk] * yk[kk];
                        }
                        cP += __popc(mp);
                    }
                }
                for (int c = 0; c < 6; ++c) {
                    const double yc = __shfl_sync(full, yv, c);
                    if (lane < 6 && lane > c) yv -= Lr[c] * yc;
                }
                if (lane < 6) vec[6 * p + lane] = yv;
                __syncwarp();
            }
            const int done = chunk == 0 ? 4 : 4 + 5 * chunk;
            if (done >= nb) break;
        }
    }
    // backward substitution, descending blocks
    for (int p = k - 1; p >= 0; --p) {
        double xv = 0.0;
        if (lane < 6) {
            xv = vec[6 * p + lane] / Dg[36LL * p + 7 * lane];
            const unsigned* cp = colm + (size_t)p * W;
            for (int w = W - 1; w >= 0; --w) {
                unsigned mm = cp[w];
                while (mm) {
                    const int bb = 31 - __clz(mm);
                    mm &= ~(1u << bb);
                    const int I = 32 * w + bb;
                    const double* Lip = Lv + 36LL * (rowptr[I] + mask_rank(rowm + (size_t)I * W, p));
                    const double* xi = vec + 6 * I;
                    for (int r = 5; r >= 0; --r) xv -= Lip[6 * r + lane] * xi[r];
                }
            }
        }
        for (int c = 5; c >= 0; --c) {
            const double xc = __shfl_sync(full, xv, c);
            if (lane < c) xv -= Dg[36LL * p + 6 * c + lane] * xc;
        }
        if (lane < 6) vec[6 * p + lane] = xv;
        __syncwarp();
    }
    for (int e = lane; e < 6 * k; e += 32) S.dx[6 * body_at[e / 6] + e % 6] = vec[e];
    __syncwarp();
    return 0;
}

// ---------------------------------------------------------------------------
// Grid-wide execution of the Newton solve: G co-resident CTAs (cooperative
// launch, G a power of two), one counting barrier in global memory with a
// bounded wait.  G = 1 degenerates to __syncthreads.
// ---------------------------------------------------------------------------
constexpr int kNewtonThreads = 512;
constexpr int kNewtonSlabBytes = 11 * 1024;   // per warp: a chain-sized component factors in shared memory
constexpr int kNewtonDynSmem = (kNewtonThreads / 32) * kNewtonSlabBytes;
constexpr int kMaxNewtonGrid = 64;
constexpr unsigned kBarrierSpinLimit = 1u << 24;   // x >= 64 ns sleeps: about a second

// arrival of a grid barrier: an acq_rel fence at GPU scope (cumulative over
// the writes this thread has observed, i.e. its CTA's writes before the
// preceding __syncthreads), then a relaxed add without a return value
__device__ __forceinline__ void red_release_add_u32(unsigned* p, unsigned v) {
    asm volatile("fence.acq_rel.gpu;\n\tred.relaxed.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// The cluster form: when the G CTAs are one thread-block cluster (G <= 16 on
// sm_100), a grid barrier is the cluster's hardware barrier, with release /
// acquire semantics at cluster scope (about 0.26 us against about 1.1 us for
// the global-memory barrier on a B200).  All CTAs of the kernel take the same
// branches (every decision reads grid-reduced values), so every thread
// arrives at every barrier.
__device__ __forceinline__ unsigned cluster_ctas() {
    unsigned n;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(n));
    return n;
}
__device__ __forceinline__ void cluster_barrier() {
    asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
}

struct GridCtx {
    int G, b, gtid, gthreads;
    bool cluster;         // the G CTAs form one cluster: hardware barrier
    int lin;              // element index of this thread in NX_GRID_FOR: CTA-interleaved
    unsigned* count;      // arrivals, zeroed before each launch
    int* abort;           // set by a CTA whose wait ran out
    int* status;
    unsigned target;
    unsigned limit;       // polls before a wait gives up
    int* sh_ok;           // shared: 0 once this CTA has given up
    __device__ bool sync() {
        if (G == 1) { __syncthreads(); return true; }
        if (cluster) { cluster_barrier(); return true; }
        target += G;
        __syncthreads();
        if (threadIdx.x == 0) {
            int ok = *sh_ok;
            if (ok) {
                // release the CTA's writes, then poll with acquire loads
                red_release_add_u32(count, 1u);
                unsigned spins = 0;
                while (ld_acquire_u32(count) < target) {
                    ++spins;
                    if (spins > limit || ((spins & 63u) == 0 && *(volatile int*)abort)) {
                        ok = 0;
                        atomicExch(abort, 1);
                        atomicExch(status, NXD_TIMEOUT);
                        break;
                    }
                    if (spins > 32) __nanosleep(64);
                }
            }
            *sh_ok = ok;
        }
        __syncthreads();
        return *sh_ok != 0;
    }
};

// Fixed-tree sums over the grid: CTA b reduces the residue class b mod G
// (elements b + G m) with the block scheme, the G class sums go through
// global memory once (one barrier), every CTA finishes the last log2 G
// levels itself.  Same double as the plain loop over the padded length.
struct GridRed {
    GridCtx* gc;
    double* sh;           // shared: kRedMaxQ * 32
    double* part;         // global: 2 * kRedMaxQ * stride
    int parity;
    int stride;           // partials per reduction slot: >= G
    template <int Q, typename F>
    __device__ void sums(const int (&n)[Q], F f, double (&out)[Q]) {
        static_assert(Q <= kRedMaxQ, "too many simultaneous reductions");
        const int G = gc->G, b = gc->b, B = blockDim.x, nw = B >> 5;
        const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
        double* gp = part + parity * (kRedMaxQ * stride);
        parity ^= 1;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const double v = warp_tree(lane_fold(n[q], b + G * (w + nw * l), G * B, [&](int e) { return f(q, e); }));
            if (l == 0) sh[q * 32 + w] = v;
        }
        __syncthreads();
        if (w == 0) {
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const double t = warp_tree(l < nw ? sh[q * 32 + l] : 0.0);
                if (l == 0) { if (G == 1) sh[q * 32] = t; else gp[q * stride + b] = t; }
            }
        }
        gc->sync();
        if (G == 1) {
#pragma unroll
            for (int q = 0; q < Q; ++q) out[q] = sh[q * 32];
            __syncthreads();
            return;
        }
#pragma unroll
        for (int q = 0; q < Q; ++q)
            out[q] = warp_tree(lane_fold(G, l, 32, [&](int e) { return __ldcg(gp + q * stride + e); }));
    }
    __device__ double max(double v) {
        const int G = gc->G, b = gc->b;
        for (int o = 16; o > 0; o >>= 1) v = dmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        double* gp = part + parity * (kRedMaxQ * stride);
        parity ^= 1;
        if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
        __syncthreads();
        if (threadIdx.x < 32) {
            double w = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
            for (int o = 16; o > 0; o >>= 1) w = dmax(w, __shfl_xor_sync(0xffffffffu, w, o));
            if (threadIdx.x == 0) { if (G == 1) sh[0] = w; else gp[b] = w; }
        }
        gc->sync();
        if (G == 1) { const double r = sh[0]; __syncthreads(); return r; }
        double w = 0.0;
        for (int e = threadIdx.x & 31; e < G; e += 32) w = dmax(w, __ldcg(gp + e));
        for (int o = 16; o > 0; o >>= 1) w = dmax(w, __shfl_xor_sync(0xffffffffu, w, o));
        return w;
    }
};

// grid-strided loop over [0, n)
// Grid-stride loop with consecutive elements on consecutive CTAs (element e
// on CTA e mod G), so that short lists of heavy elements (joints, bodies)
// spread over all SMs instead of filling the first CTAs.
#define NX_GRID_FOR(e, n, gc) for (int e = (gc).lin; e < (n); e += (gc).gthreads)

// poses (and the x <- xt copy after an accepted step) for every body
__device__ void grid_poses(const Solver& S, const double* x, const GridCtx& gc) {
    NX_GRID_FOR(i, S.N, gc) {
        const Q q0 = ldq(S.quat0 + 4 * i);
        const V3 th = xs3(x, 6 * i + 3);
        stq(S.qj + 4 * i, rot_joint(q0, th));
        stq(S.qg + 4 * i, rot_gt(q0, th));
    }
}

// computeValue and computeContactValue at x from one set of fixed-tree sums;
// poses at x and the drives' value call must be done.
__device__ void grid_energies(const Solver& S, const double* x, double s, int C, GridRed& R, double& full,
                              double& contact) {
    const bool bar = *S.barrier_in_forms_ptr != 0, fr = *S.friction_form_ptr != 0;
    const double dh = *S.bdhat_ptr, kap = *S.bkappa_ptr;
    const int n[5] = {S.N, S.N, S.J, bar ? C : 0, fr ? C : 0};
    double sum[5];
    R.sums<5>(n, [&](int q, int e) -> double {
        switch (q) {
            case 0: return inertia_value(S, e, x);
            case 1: return gravity_value(S, e, x);
            case 2: { double Cj[6]; const int dim = joint_residual(S, e, x, Cj, nullptr); return joint_energy(S, e, Cj, dim); }
            case 3: return barrier_value(contact_distance(S.contacts[e], x), dh, kap);
            default: return friction_value(S, e, x);
        }
    }, sum);
    double v = sum[0];
    v += s * sum[1];
    v += sum[2];
    for (int d = 0; d < S.D; ++d) v += s * S.dE[d];
    if (S.D > 0) R.gc->sync();   // dE is rewritten by the next value call
    double c = 0.0;
    if (bar) { v += s * sum[3]; c += s * sum[3]; }
    if (fr) { v += s * sum[4]; c += s * sum[4]; }
    full = v;
    contact = c;
}

// 6x6 LDL^T solve of body i's diagonal block (a body no item couples)
__device__ __forceinline__ void solve_singleton(const Solver& S, int i) {
    double A[36], b[6];
#pragma unroll
    for (int e = 0; e < 36; ++e) A[e] = S.Hd[36 * i + e];
#pragma unroll
    for (int e = 0; e < 6; ++e) b[e] = -S.g[6 * i + e];
    if (!ldlt6_solve(A, b)) { atomicExch(S.solve_fail, 1); return; }
#pragma unroll
    for (int e = 0; e < 6; ++e) S.dx[6 * i + e] = b[e];
}

// Solve H dx = -g over the grid.  Returns false (all threads) on failure.
// The block structure (components, their member and item lists, each
// component's elimination order and fill pattern) depends only on which
// coupling items are active.  `cached` says an earlier call of this launch
// built it; it is reused, after one grid reduction over the items' states,
// when no item changed state since.  A component's own symbolic part is
// reused when its warp's shared slab still holds it (one component per warp).
__device__ bool grid_solve(const Solver& S, double s, int C, GridCtx& gc, GridRed& R, int* sh_scan, int* sh_flag,
                           int* sh_wcomp, bool& cached) {
    const int N = S.N;
    const int n_items = S.ext_n >= 0 ? S.ext_n : S.J + S.D + 2 * C;
    bool reuse = false;
    if (cached) {
        if (gc.gtid == 0) { *S.mpool_off = 0; *S.pool_off = 0; *S.solve_fail = 0; }
        double ch = 0.0;
        NX_GRID_FOR(it, n_items, gc) if ((item_active(S, it) ? 1 : 0) != S.iact[it]) ch = 1.0;
        reuse = R.max(ch) == 0.0;
    }
    if (reuse) {
        NX_GRID_FOR(i, N, gc) {
            if (S.comp[i] != i || S.rflag[i + 1] != S.rflag[i]) continue;
            solve_singleton(S, i);
        }
        NX_PHASE(3);
    } else {
    NX_GRID_FOR(i, N + 1, gc) {
        if (i < N) S.parent[i] = i;
        S.mcnt[i] = 0; S.icnt[i] = 0; S.rflag[i] = 0;
    }
    if (gc.gtid == 0) { *S.comp_next = 0; *S.mpool_off = 0; *S.pool_off = 0; *S.solve_fail = 0; }
    gc.sync();
    NX_GRID_FOR(it, n_items, gc) {
        const bool act = item_active(S, it);
        S.iact[it] = act ? 1 : 0;
        if (!act) continue;
        int a, b;
        item_bodies(S, it, a, b);
        if (a != b) uf_union(S.parent, a, b);
    }
    gc.sync();
    NX_GRID_FOR(i, N, gc) {
        const int r = uf_find(S.parent, i);
        S.comp[i] = r;
        atomicAdd(&S.mcnt[r], 1);
    }
    NX_GRID_FOR(it, n_items, gc) {
        if (!S.iact[it]) continue;
        int a, b;
        item_bodies(S, it, a, b);
        if (a != b) atomicAdd(&S.icnt[uf_find(S.parent, a)], 1);
    }
    gc.sync();
    // singletons: one thread each, in registers
    NX_GRID_FOR(i, N, gc) {
        const bool multi = S.comp[i] == i && S.mcnt[i] >= 2;
        S.rflag[i] = multi ? 1 : 0;
        if (S.comp[i] != i || S.mcnt[i] != 1) continue;
        solve_singleton(S, i);
    }
    gc.sync();
    NX_PHASE(3);
    if (gc.b == 0) {
        for (int i = threadIdx.x; i < N; i += blockDim.x)
            if (!S.rflag[i]) S.mcnt[i] = 0;
        __syncthreads();
        int* const arr[3] = {S.mcnt, S.icnt, S.rflag};
        block_scan_excl<3>(arr, N, sh_scan);
    }
    gc.sync();
    NX_GRID_FOR(r, N, gc) {
        if (S.rflag[r + 1] != S.rflag[r]) S.comp_root[S.rflag[r]] = r;
        S.local[r] = 0;    // member cursor per root
        S.parent[r] = 0;   // item cursor per root
    }
    gc.sync();
    NX_GRID_FOR(i, N, gc) {
        const int r = S.comp[i];
        if (S.mcnt[r + 1] - S.mcnt[r] >= 2) S.members[S.mcnt[r] + atomicAdd(&S.local[r], 1)] = i;
    }
    NX_GRID_FOR(it, n_items, gc) {
        if (!S.iact[it]) continue;
        int a, b;
        item_bodies(S, it, a, b);
        if (a == b) continue;
        const int r = S.comp[a];
        S.items[S.icnt[r] + atomicAdd(&S.parent[r], 1)] = it;
    }
    gc.sync();
    NX_PHASE(3);
    }
    const int n_comp = __ldcg(S.rflag + N);
    // multi-body components: one warp each, consecutive components on
    // consecutive CTAs (warp w of CTA b takes components w G + b, + G nw, ...)
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nwarps = gc.G * (blockDim.x >> 5);
    const bool one_each = n_comp <= nwarps;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned char* const slab = S.slab_bytes > 0 ? smem_raw + (size_t)w * S.slab_bytes : nullptr;
    for (int o = w * gc.G + gc.b; o < n_comp; o += nwarps) {
        bool in_slab = false;
        const int rc = solve_component(S, S.comp_root[o], s, C, slab, reuse && one_each && sh_wcomp[w] == o, in_slab);
        if (lane == 0) sh_wcomp[w] = (rc == 0 && in_slab) ? o : -1;
        if (rc != 0 && lane == 0) {
            atomicExch(S.solve_fail, 1);
            if (rc == 2) atomicExch(S.status, NXD_CAPACITY);
        }
    }
    gc.sync();
    cached = true;
    NX_PHASE(4);
    if (threadIdx.x == 0) *sh_flag = __ldcg(S.solve_fail);
    __syncthreads();
    const bool fail = *sh_flag != 0;
    __syncthreads();
    return !fail;
}

// ---------------------------------------------------------------------------
// The kernel: one ALM iteration's Newton solve + joint bookkeeping, on G
// co-resident CTAs (every branch below depends only on grid-reduced values,
// so all CTAs take the same path and meet at every barrier).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void newton_body(const Solver& S) {
    __shared__ unsigned long long sh_keys[kMaxIncidence];
    __shared__ double sh_red[kRedMaxQ * 32];
    __shared__ int sh_scan[3 * 32];
    __shared__ int sh_flag, sh_ok;
    __shared__ int sh_wcomp[kNewtonThreads / 32];   // component whose structure each warp's slab holds
    if (*S.alm_done) return;
    if (threadIdx.x < kNewtonThreads / 32) sh_wcomp[threadIdx.x] = -1;
    NX_PHASE_START();
    GridCtx gc;
    gc.G = gridDim.x; gc.b = blockIdx.x;
    gc.gtid = blockIdx.x * blockDim.x + threadIdx.x; gc.gthreads = gridDim.x * blockDim.x;
    gc.lin = threadIdx.x * gc.G + gc.b;
    gc.count = S.bar_count; gc.abort = S.bar_abort; gc.status = S.status; gc.target = 0; gc.sh_ok = &sh_ok;
    gc.cluster = gc.G > 1 && (int)cluster_ctas() == gc.G;
    gc.limit = S.spin_limit ? S.spin_limit : kBarrierSpinLimit;
    if (threadIdx.x == 0) sh_ok = 1;
    __syncthreads();
    if (S.dbg_hold && gc.G > 1 && !gc.cluster && gc.b == gc.G - 1) {
        // failure-detection hook (nxd_debug_grid_wait): this CTA keeps away
        // from the first barrier until the others have given up on it, or
        // for at most 64 x limit polls
        if (threadIdx.x == 0)
            for (unsigned k = 0; k < 64u * gc.limit && !*(volatile int*)gc.abort; ++k) __nanosleep(64);
        __syncthreads();
    }
    GridRed R;
    R.gc = &gc; R.sh = sh_red; R.part = S.gpart; R.parity = 0; R.stride = kMaxNewtonGrid;
    const int N = S.N;
    const int C = *S.ncontacts_ptr;
    const double s = *S.scale_ptr;   // ImplicitTimeIntegrator::acceleration_scaling
    const int n6 = 6 * N;
    const bool bar = *S.barrier_in_forms_ptr != 0, fr = *S.friction_form_ptr != 0;
    const double dh = *S.bdhat_ptr;
    if (gc.b == 0) {
        build_contact_incidence(S, C, sh_keys);
        if (threadIdx.x == 0) *S.n_heavy = 0;
        __syncthreads();
        for (int i = threadIdx.x; i < N; i += blockDim.x) {
            const bool h = S.cinc_off[i + 1] - S.cinc_off[i] > kHeavyEnds;
            S.heavy[i] = h ? 1 : 0;
            if (h) S.heavy_list[atomicAdd(S.n_heavy, 1)] = i;
        }
    }
    if (!gc.sync()) return;
    NX_PHASE(0);
    // heavy bodies' DOFs: one warp each (any order: each DOF is independent);
    // the incidence keys are dead from here on, their shared memory holds
    // each warp's 256 doubles of contact terms
    const int n_heavy = __ldcg(S.n_heavy);
    double* const tw = reinterpret_cast<double*>(sh_keys) + 256 * (threadIdx.x >> 5);
    const int hwarp = (threadIdx.x >> 5) * gc.G + gc.b, hwarps = gc.G * (blockDim.x >> 5);

    bool converged = false, poses_at_x = false, aborted = false;
    // energies at the accepted iterate: the next line search's starting
    // values are the same function of the same x, so they are reused when no
    // stateful form (a velocity drive) has to see its value call
    bool have_fx = false, cached = false;
    double fx_acc = 0.0, fc_acc = 0.0;
    int iters = 0;
    for (int iter = 0; iter < S.newton_max_iters; ++iter) {
        iters = iter;
        // gradient at x (drives: gradient call)
        if (!poses_at_x) grid_poses(S, S.x, gc);
        poses_at_x = true;
        NX_GRID_FOR(d, S.D, gc) drive_eval(S, d, S.x, 1);
        if (!gc.sync()) { aborted = true; break; }
        NX_GRID_FOR(e, S.J + C, gc) {
            if (e < S.J) { joint_eval(S, e, S.x, true); continue; }
            const int c = e - S.J;
            if (bar) barrier_eval(S, c, S.x);
            if (fr) friction_eval(S, c, S.x, true);
        }
        if (!gc.sync()) { aborted = true; break; }
        double gm = 0.0;
        NX_GRID_FOR(e, n6, gc) {
            if (n_heavy > 0 && S.heavy[e / 6]) continue;
            double g, cg;
            gradient_dof(S, S.x, s, e / 6, e % 6, bar, fr, dh, g, cg);
            S.g[e] = g;
            S.cg[e] = cg;
            gm = dmax(gm, fabs(g));
        }
        for (int t = hwarp; t < 6 * n_heavy; t += hwarps) {
            const int i = S.heavy_list[t / 6], k = t % 6;
            double g, cg;
            gradient_dof_warp(S, S.x, s, i, k, bar, fr, dh, g, cg, tw);
            if ((threadIdx.x & 31) == 0) { S.g[6 * i + k] = g; S.cg[6 * i + k] = cg; }
            gm = dmax(gm, fabs(g));
        }
        gm = R.max(gm);
        NX_PHASE(1);
        if (gm < S.newton_tol) { converged = true; break; }
        // Hessian (drives: hessian call)
        if (S.D > 0) {
            NX_GRID_FOR(d, S.D, gc) drive_eval(S, d, S.x, 2);
            gc.sync();
        }
        {
            const bool b2 = bar, f2 = fr;
            NX_GRID_FOR(e, n6, gc) {
                if (n_heavy > 0 && S.heavy[e / 6]) continue;
                double H[6];
                diag_hessian_row(S, s, e / 6, e % 6, b2, f2, dh, H);
                for (int k = 0; k < 6; ++k) S.Hd[6 * e + k] = H[k];
            }
            for (int t = hwarp; t < 6 * n_heavy; t += hwarps) {
                const int e = 6 * S.heavy_list[t / 6] + t % 6;
                double H[6];
                diag_hessian_row_warp(S, s, e / 6, e % 6, b2, f2, dh, H, tw);
                if ((threadIdx.x & 31) == 0)
                    for (int k = 0; k < 6; ++k) S.Hd[6 * e + k] = H[k];
            }
        }
        if (!gc.sync()) { aborted = true; break; }
        NX_PHASE(2);
        if (!grid_solve(S, s, C, gc, R, sh_scan, &sh_flag, sh_wcomp, cached)) break;
        // line search (max step 1): the value calls at x, then descent terms
        if (S.D > 0) {
            NX_GRID_FOR(d, S.D, gc) drive_eval(S, d, S.x, 0);
            gc.sync();
        }
        double fx, fc, descent, cdesc;
        {
            if (have_fx) { fx = fx_acc; fc = fc_acc; }
            else grid_energies(S, S.x, s, C, R, fx, fc);
            const int nn[2] = {n6, n6};
            double dd[2];
            R.sums<2>(nn, [&](int q, int e) { return (q == 0 ? S.g[e] : S.cg[e]) * S.dx[e]; }, dd);
            descent = dd[0];
            cdesc = dd[1];
        }
        NX_PHASE(5);
        if (descent > 0) { if (gc.gtid == 0) atomicAdd(S.ls_fail, 1); poses_at_x = true; break; }
        double alpha = 1.0;
        bool done = false;
        for (int ls = 0; ls < S.ls_max_iters; ++ls) {
            NX_GRID_FOR(i, N, gc) {
                for (int k = 0; k < 6; ++k) S.xt[6 * i + k] = S.x[6 * i + k] + alpha * S.dx[6 * i + k];
                const Q q0 = ldq(S.quat0 + 4 * i);
                const V3 th = xs3(S.xt, 6 * i + 3);
                stq(S.qj + 4 * i, rot_joint(q0, th));
                stq(S.qg + 4 * i, rot_gt(q0, th));
            }
            NX_GRID_FOR(d, S.D, gc) drive_eval(S, d, S.xt, 0);
            gc.sync();
            double fn, fcn;
            grid_energies(S, S.xt, s, C, R, fn, fcn);
            const bool cok = cdesc <= 0.0 ? (fcn <= fc + S.ls_c1 * alpha * cdesc) : (fcn <= fc);
            if (fn <= fx + S.ls_c1 * alpha * descent && cok) { done = true; fx_acc = fn; fc_acc = fcn; break; }
            alpha *= S.ls_rho;
        }
        NX_PHASE(6);
        if (!done) { if (gc.gtid == 0) atomicAdd(S.ls_fail, 1); poses_at_x = false; break; }
        // accept: x <- xt (each body by the thread that posed it)
        NX_GRID_FOR(i, N, gc)
            for (int k = 0; k < 6; ++k) S.x[6 * i + k] = S.xt[6 * i + k];
        poses_at_x = true;
        have_fx = S.D == 0;
        if (S.D > 0) gc.sync();   // the drives' next gradient call reads any body's x
        if (iter == S.newton_max_iters - 1) iters = S.newton_max_iters;
    }
    if (aborted) return;
    if (gc.gtid == 0) {
        atomicAdd(S.newton_iters, iters);
        *S.converged = converged ? 1 : 0;
    }
    // ALM: violation, hardening, lambda update (IPCSolver.cpp:1084-1110);
    // each joint hardens with its own pre-update stiffness, then takes
    // lambda += mu_new C
    if (!poses_at_x) grid_poses(S, S.x, gc);
    if (!gc.sync()) return;
    double mcv = 0.0, dual = 0.0;
    NX_GRID_FOR(j, S.J, gc) {
        double Cj[6];
        const int dim = joint_residual(S, j, S.x, Cj, nullptr);
        for (int k = 0; k < 6; ++k) S.jC[6 * j + k] = Cj[k];
        double inf = 0.0;
        for (int k = 0; k < dim; ++k) inf = dmax(inf, fabs(Cj[k]));
        mcv = dmax(mcv, inf);
        double mu = S.jmu[j];
        const double dc = mu * inf;
        if (isfinite(dc)) dual = dmax(dual, dmin(dc, 1e12));
        else dual = dmax(dual, 1e12);
        if (inf > S.alm_hardening_trigger * S.alm_constraint_tol) {
            const double ns = mu * S.alm_hardening_ratio;
            mu = isfinite(ns) ? dmin(ns, 1e12) : 1e12;
            S.jmu[j] = mu;
        }
        double* lam = S.jlam + 6 * j;
        if (joint_is_limit(S.jtype[j])) for (int k = 0; k < dim; ++k) lam[k] = dmax(0.0, lam[k] + mu * Cj[k]);
        else for (int k = 0; k < dim; ++k) lam[k] += mu * Cj[k];
    }
    mcv = R.max(mcv);
    dual = R.max(dual);
    if (gc.gtid == 0) {
        *S.alm_mcv = mcv;
        *S.alm_dual = dual;
    }
    NX_PHASE(7);
#ifdef NXD_PHASE_TIMERS
    if (gc.gtid == 0)
        printf("PH G=%d C=%d it=%d init=%lld grad=%lld hess=%lld symb=%lld comp=%lld ls0=%lld ls=%lld post=%lld\n", gc.G, C,
               iters, nx_ph_acc[0], nx_ph_acc[1], nx_ph_acc[2], nx_ph_acc[3], nx_ph_acc[4], nx_ph_acc[5], nx_ph_acc[6],
               nx_ph_acc[7]);
#endif
}
constexpr int kLB_newton = kNewtonThreads;
__global__ void __launch_bounds__(kNewtonThreads) k_newton(const __grid_constant__ Solver S) { newton_body(S); }

// ---------------------------------------------------------------------------
// LinearSolver::analyzePattern + factorize + solve (LinearSolver.cpp:11-39) for
// a caller's block matrix: diagonal blocks summed in storage order into Hd,
// the right-hand side as -g, then the Newton solve's component LDL^T on one
// CTA (the lower triangle in elimination order, as SimplicialLDLT's Lower).
// ---------------------------------------------------------------------------
__global__ void k_bsr_prepare(Solver S, const int* row_ptr, const double* b, int* ext_row) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.N) return;
    double H[36];
    for (int e = 0; e < 36; ++e) H[e] = 0.0;
    for (int k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
        ext_row[k] = i;
        if (S.ext_col[k] == i)
            for (int e = 0; e < 36; ++e) H[e] += S.ext_vals[36LL * k + e];
    }
    for (int e = 0; e < 36; ++e) S.Hd[36 * i + e] = H[e];
    for (int k = 0; k < 6; ++k) S.g[6 * i + k] = -b[6 * i + k];
}
__global__ void __launch_bounds__(kNewtonThreads) k_linear_solve(const __grid_constant__ Solver S) {
    __shared__ double sh_red[kRedMaxQ * 32];
    __shared__ int sh_scan[3 * 32];
    __shared__ int sh_flag, sh_ok;
    __shared__ int sh_wcomp[kNewtonThreads / 32];
    if (threadIdx.x < kNewtonThreads / 32) sh_wcomp[threadIdx.x] = -1;
    if (threadIdx.x == 0) sh_ok = 1;
    GridCtx gc;
    gc.G = 1; gc.b = 0; gc.gtid = threadIdx.x; gc.gthreads = blockDim.x; gc.lin = threadIdx.x;
    gc.count = S.bar_count; gc.abort = S.bar_abort; gc.status = S.status; gc.target = 0; gc.sh_ok = &sh_ok;
    gc.cluster = false; gc.limit = kBarrierSpinLimit;
    __syncthreads();
    GridRed R;
    R.gc = &gc; R.sh = sh_red; R.part = S.gpart; R.parity = 0; R.stride = kMaxNewtonGrid;
    bool cached = false;
    grid_solve(S, 1.0, 0, gc, R, sh_scan, &sh_flag, sh_wcomp, cached);
}

}  // namespace nx
