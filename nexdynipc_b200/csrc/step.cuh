// step.cuh — per-step bookkeeping kernels of IPCSolver::step
// (src/Dynamics/IPCSolver.cpp:808-1231) around the geometry and Newton
// kernels: adaptive-barrier initialisation and stiffness update, integrator
// set-up, contact-form installation, the ALM convergence test, the 2000
// contact cap and the state write-back.
#pragma once

#include "solver.cuh"

namespace nx {

// Device-resident scalars of one context.
struct Scalars {
    double dhat;            // AdaptiveBarrier::currentDhat
    double kappa;           // AdaptiveBarrier::currentStiffness
    double dt;              // step dt (computeMaxStep result)
    double scale;           // ImplicitTimeIntegrator::acceleration_scaling
    double friction_mu;     // FrictionForm coefficient of this step
    double bdhat, bkappa;   // DistanceBarrierForm parameters
    double bmd;             // estimateBroadPhaseMinDistance(2 dhat)
    double md;              // computeSceneMinDistance (pruned)
    double md_radius;       // half the widest pruning band
    double alm_mcv, alm_dual, alm_cres;
    double last_vw, last_tsat;
    int barrier_initialized;
    int md_gate;
    int alm_done;
    int barrier_form, barrier_in_forms, friction_form;
    int n_pairs, n_md_pairs;
    int fv_items, ee_items, vv_items;
    int fv_hits, ee_hits, vv_hits;
    int zero_hits;          // 1 when FV+EE produced nothing (VV fallback runs)
    int n_contacts, n_contacts_raw;
    int nnf;
    int status;
    int newton_iters, converged, ls_fail, alm_iters;
    int n_pairs_overflow;
};

struct StepCfg {
    int N, D;
    int enable_adaptive, enable_friction;
    double friction_coeff;
    double alm_constraint_tol, alm_dual_tol, alm_contact_tol;
    int newmark;            // 1: ImplicitNewmark(beta, gamma), 0: ImplicitEuler
    double beta, gamma;
};

// IPCSolver::initializeAdaptiveBarrier (IPCSolver.cpp:327-353) +
// AdaptiveBarrier::initialize (AdaptiveBarrier.h:27-31); runs once per context.
__device__ __forceinline__ void barrier_init_body(const StepCfg& cfg, const double* mass, const double* pos, Scalars* sc) {
    __shared__ double bb[6];
    NX_BLOCK_RED(R);
    if (!cfg.enable_adaptive || sc->barrier_initialized || cfg.N == 0) return;
    const double tm = R.sum(cfg.N, [&](int i) { return mass[i]; });
    // scene bounds: per-thread, per-warp, then across warps (min / max are
    // exact; a +-0 tie only changes the sign of a zero, which mx - mn absorbs)
    __shared__ double wb[32 * 6];
    V3 mn = v3(INFINITY, INFINITY, INFINITY), mx = v3(-INFINITY, -INFINITY, -INFINITY);
    for (int i = threadIdx.x; i < cfg.N; i += blockDim.x) { mn = cwmin(mn, ld3(pos + 3 * i)); mx = cwmax(mx, ld3(pos + 3 * i)); }
    for (int o = 16; o > 0; o >>= 1) {
        mn = cwmin(mn, v3(__shfl_xor_sync(0xffffffffu, mn.x, o), __shfl_xor_sync(0xffffffffu, mn.y, o), __shfl_xor_sync(0xffffffffu, mn.z, o)));
        mx = cwmax(mx, v3(__shfl_xor_sync(0xffffffffu, mx.x, o), __shfl_xor_sync(0xffffffffu, mx.y, o), __shfl_xor_sync(0xffffffffu, mx.z, o)));
    }
    if ((threadIdx.x & 31) == 0) { st3(wb + 6 * (threadIdx.x >> 5), mn); st3(wb + 6 * (threadIdx.x >> 5) + 3, mx); }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) { mn = cwmin(mn, ld3(wb + 6 * w)); mx = cwmax(mx, ld3(wb + 6 * w + 3)); }
        st3(bb, mn); st3(bb + 3, mx);
        const double am = tm / (double)cfg.N;
        double diag = norm(mx - mn);
        if (diag < 1e-6) diag = 1.0;
        sc->kappa = 1e11 * am / (diag * diag);
        sc->dhat = 1e-3;
        sc->barrier_initialized = 1;
    }
}
constexpr int kLB_barrier_init = kSolverThreads;
__global__ void __launch_bounds__(kSolverThreads) k_barrier_init(const __grid_constant__ StepCfg cfg, const double* mass, const double* pos, Scalars* sc) { barrier_init_body(cfg, mass, pos, sc); }

__device__ __forceinline__ void md_gate_body(Scalars* sc, const double* max_md_tol) {
    sc->md_gate = (sc->bmd < sc->dhat * 2.0) ? 1 : 0;
    sc->md = INFINITY;
    sc->md_radius = 0.5 * (kPruneBand + *max_md_tol) + 1e-12;
}
constexpr int kLB_md_gate = 0;
__global__ void k_md_gate(Scalars* sc, const double* max_md_tol) { md_gate_body(sc, max_md_tol); }

// AdaptiveBarrier::updateStiffness (AdaptiveBarrier.h:33-37)
__device__ __forceinline__ void kappa_update_body(Scalars* sc) {
    if (!sc->md_gate) return;
    const double md = sc->md;
    if (md < INFINITY && md < 1e-9 && sc->kappa < 1e20) sc->kappa = dmin(sc->kappa * 2.0, 1e20);
}
constexpr int kLB_kappa_update = 0;
__global__ void k_kappa_update(Scalars* sc) { kappa_update_body(sc); }

// Integrator init / x_tilde (IPCSolver.cpp:839-861, ImplicitEulerIntegrator.cpp:5-11),
// contact-form flags (IPCSolver.cpp:873-921) and drive set-up (IPCSolver.cpp:923-958).
__device__ __forceinline__ void step_setup_body(const StepCfg& cfg, double dt, const double* pos, const double* quat, const double* vel, const double* omega, const double* lacc, const double* aacc, double* x, double* xhat, double* xprev, double* vprev, double* aprev, double* pos0, double* quat0, Scalars* sc, const Drv* dprm, double* dfilt, int* dfinit, int* dhas_prev) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < cfg.N) {
        for (int k = 0; k < 3; ++k) {
            const double p = pos[3 * i + k];
            xprev[6 * i + k] = p; xprev[6 * i + 3 + k] = 0.0;
            vprev[6 * i + k] = vel[3 * i + k]; vprev[6 * i + 3 + k] = omega[3 * i + k];
            aprev[6 * i + k] = lacc[3 * i + k]; aprev[6 * i + 3 + k] = aacc[3 * i + k];
            pos0[3 * i + k] = p;
        }
        for (int k = 0; k < 4; ++k) quat0[4 * i + k] = quat[4 * i + k];
        // x_tilde: ImplicitEuler (ImplicitEulerIntegrator.cpp:5-7) or
        // ImplicitNewmark (ImplicitNewmark.cpp:8-10), Eigen's evaluation order
        const double s1 = (dt * dt) * (0.5 - cfg.beta);
        for (int k = 0; k < 6; ++k) {
            double xh = xprev[6 * i + k] + dt * vprev[6 * i + k];
            if (cfg.newmark) xh = xh + s1 * aprev[6 * i + k];
            xhat[6 * i + k] = xh;
            x[6 * i + k] = xh;
        }
    }
    if (i < cfg.D) {
        const Drv& p = dprm[i];
        if (p.tau <= 0.0) { dfilt[i] = p.vt; dfinit[i] = 0; }
        else if (!dfinit[i]) { dfilt[i] = p.vt; dfinit[i] = 1; }
        else if (dt > 0.0) { const double al = dt / (p.tau + dt); dfilt[i] += al * (p.vt - dfilt[i]); }
        dhas_prev[i] = 0;
    }
    if (i == 0) {
        sc->dt = dt;
        sc->scale = cfg.newmark ? (cfg.beta * dt) * dt : dt * dt;
        sc->friction_mu = cfg.friction_coeff;
        const bool needs = cfg.enable_adaptive || (cfg.enable_friction && cfg.friction_coeff > 0.0);
        sc->barrier_form = needs ? 1 : 0;
        sc->barrier_in_forms = (cfg.enable_adaptive && needs) ? 1 : 0;
        sc->friction_form = (cfg.enable_friction && cfg.friction_coeff > 0.0) ? 1 : 0;
        sc->bdhat = dmax(1e-9, sc->dhat);
        sc->bkappa = dmax(0.0, sc->kappa);
        sc->nnf = 0;
        sc->alm_done = 0;
        sc->newton_iters = 0;
        sc->ls_fail = 0;
        sc->alm_iters = 0;
        sc->converged = 0;
        sc->alm_mcv = 0.0; sc->alm_dual = 0.0; sc->alm_cres = 0.0;
    }
}
constexpr int kLB_step_setup = 0;
__global__ void k_step_setup(const __grid_constant__ StepCfg cfg, double dt, const double* pos, const double* quat, const double* vel, const double* omega, const double* lacc, const double* aacc, double* x, double* xhat, double* xprev, double* vprev, double* aprev, double* pos0, double* quat0, Scalars* sc, const Drv* dprm, double* dfilt, int* dfinit, int* dhas_prev) { step_setup_body(cfg, dt, pos, quat, vel, omega, lacc, aacc, x, xhat, xprev, vprev, aprev, pos0, quat0, sc, dprm, dfilt, dfinit, dhas_prev); }

// Friction coefficient of the step with per-pair overrides
// (IPCSolver.cpp:891-911): the mean over the active contacts of each
// contact's pair override, else the global coefficient, summed in contact
// order.  Runs only when overrides exist.
__device__ __forceinline__ void friction_mu_body(const StepCfg& cfg, Scalars* sc, const ContactRec* contacts,
                                                 const unsigned long long* keys, const double* mu, int n_keys) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int n = sc->n_contacts;
    if (n <= 0) { sc->friction_mu = cfg.friction_coeff; return; }
    double sum = 0.0;
    for (int c = 0; c < n; ++c) {
        const int k = allowed_index(keys, n_keys, contacts[c].body_a, contacts[c].body_b);
        sum += (k >= 0 && mu[k] >= 0.0) ? mu[k] : cfg.friction_coeff;
    }
    sc->friction_mu = sum / (double)n;
}
constexpr int kLB_friction_mu = 0;
__global__ void k_friction_mu(const __grid_constant__ StepCfg cfg, Scalars* sc, const ContactRec* contacts,
                              const unsigned long long* keys, const double* mu, int n_keys) {
    friction_mu_body(cfg, sc, contacts, keys, mu, n_keys);
}

// Contact totals after FV + EE (+VV) passes; gates the VV fallback.
// stage 2 clears the counts (no detection this step).
__device__ __forceinline__ void contact_totals_body(Scalars* sc, int stage, const int* skip_if, int* skip_vv) {
    if (skip_if && *skip_if != 0) { if (skip_vv) *skip_vv = 1; return; }
    if (stage == 2) { sc->n_contacts = 0; sc->n_contacts_raw = 0; return; }
    if (stage == 0) {
        sc->zero_hits = (sc->fv_hits + sc->ee_hits) == 0 ? 1 : 0;
        if (skip_vv) *skip_vv = sc->zero_hits ? 0 : 1;
        if (!sc->zero_hits) sc->vv_hits = 0;
    } else {
        const int total = sc->fv_hits + sc->ee_hits + (sc->zero_hits ? sc->vv_hits : 0);
        const int raw = total < kMaxRawContacts ? total : kMaxRawContacts;
        sc->n_contacts_raw = raw;
        sc->n_contacts = raw > kMaxContacts ? kMaxContacts : raw;
    }
}
constexpr int kLB_contact_totals = 0;
__global__ void k_contact_totals(Scalars* sc, int stage, const int* skip_if, int* skip_vv) { contact_totals_body(sc, stage, skip_if, skip_vv); }

// std::sort by distance + truncation to 2000 (IPCSolver.cpp:571-577).  The
// sort is libstdc++'s introsort, which is not stable: equal distances (common:
// hinged links overlap at their hinges, distance 0) come out in the order its
// partitions leave them, which decides both the contact order the forms sum
// in and which ties survive the cut.  sel_sort_prefix_block reproduces that
// permutation over the first 2000 positions.  One CTA of 1024 threads with
// sort_smem_bytes(32) of dynamic shared memory; runs only when more than 2000
// contacts exist.
__device__ __forceinline__ void sort_contacts_body(Scalars* sc, ContactRec* c, ContactRec* tmp, double* key, int* idx,
                                                   int* gscr, int* lscr, SortRange* small, const int* skip_if) {
    if (skip_if && *skip_if != 0) return;
    const int raw = sc->n_contacts_raw;
    if (raw <= kMaxContacts) return;
    for (int i = threadIdx.x; i < raw; i += blockDim.x) {
        key[i] = c[i].distance;
        idx[i] = i;
    }
    __syncthreads();
    extern __shared__ __align__(16) unsigned char sort_slab[];
    sel_sort_prefix_block(SelView{idx, key, gscr, lscr}, raw, kMaxContacts, small, sort_slab);
    for (int i = threadIdx.x; i < kMaxContacts; i += blockDim.x) tmp[i] = c[idx[i]];
    __syncthreads();
    for (int i = threadIdx.x; i < kMaxContacts; i += blockDim.x) c[i] = tmp[i];
}
constexpr int kLB_sort_contacts = 0;
__global__ void k_sort_contacts(Scalars* sc, ContactRec* c, ContactRec* tmp, double* key, int* idx, int* gscr, int* lscr,
                                SortRange* small, const int* skip_if) {
    sort_contacts_body(sc, c, tmp, key, idx, gscr, lscr, small, skip_if);
}

// After the Newton solve and the detection at x_new (IPCSolver.cpp:1112-1165):
// normal forces, contact residual, ALM convergence.
__device__ __forceinline__ void alm_post_body(const Solver& S, Scalars* sc, const StepCfg& cfg, double* nforce_out) {
    __shared__ unsigned long long sh_keys[kMaxIncidence];
    NX_BLOCK_RED(R);
    if (sc->alm_done) return;
    const int C = sc->n_contacts;
    const bool bform = sc->barrier_form != 0, fform = sc->friction_form != 0;
    const bool fric = cfg.enable_friction && fform;
    if (bform || fform) {
        eval_poses(S, S.x);
        __syncthreads();
        for (int c = threadIdx.x; c < C; c += blockDim.x) barrier_eval(S, c, S.x);
        __syncthreads();
        if (fric) {
            // DistanceBarrierForm::computeNormalForces (DistanceBarrierForm.cpp:70-86)
            for (int c = threadIdx.x; c < C; c += blockDim.x) {
                double nf = 0.0;
                if (bform) {
                    const double d = S.bD[c];
                    if (d < sc->bdhat && d > 0.0) nf = fabs(barrier_gradient(d, sc->bdhat, sc->bkappa));
                }
                nforce_out[c] = nf;
            }
            if (threadIdx.x == 0) sc->nnf = C;
        }
        __syncthreads();
        if (fric)
            for (int c = threadIdx.x; c < C; c += blockDim.x) friction_eval(S, c, S.x, true);
        build_contact_incidence(S, C, sh_keys);
        // max |barrier + friction gradient| over all DOFs
        double m = 0.0;
        const double dh = sc->bdhat;
        for (int e = threadIdx.x; e < 6 * S.N; e += blockDim.x) {
            const int i = e / 6, k = e % 6;
            double cb = 0.0, cf = 0.0;
            for (int q = S.cinc_off[i]; q < S.cinc_off[i + 1]; ++q) {
                const int c = S.cinc[q] >> 1, side = S.cinc[q] & 1;
                if (bform && k < 3 && S.bD[c] < dh) {
                    const double gpv = S.bGP[c];
                    const double nk = S.contacts[c].normal[k];
                    cb += side == 0 ? (-gpv) * nk : gpv * nk;
                }
                if (fric && friction_on(S, c)) {
                    const double* Jx = (side == 0 ? S.fJA : S.fJB) + 18 * c;
                    const double* fg = S.fFG + 3 * c;
                    cf += Jx[k] * fg[0] + Jx[6 + k] * fg[1] + Jx[12 + k] * fg[2];
                }
            }
            double v = 0.0;
            if (bform) v += cb;
            if (fric) v += cf;
            m = dmax(m, fabs(v));
        }
        m = R.max(m);
        if (threadIdx.x == 0) sc->alm_cres = isfinite(m) ? m : 1e12;
    } else if (threadIdx.x == 0) {
        sc->alm_cres = 0.0;
    }
    if (threadIdx.x == 0) {
        sc->alm_mcv = *S.alm_mcv;
        sc->alm_dual = *S.alm_dual;
        sc->alm_iters += 1;
        if (*S.converged && sc->alm_mcv <= cfg.alm_constraint_tol && sc->alm_dual <= cfg.alm_dual_tol &&
            sc->alm_cres <= cfg.alm_contact_tol)
            sc->alm_done = 1;
    }
}
constexpr int kLB_alm_post = kSolverThreads;
__global__ void __launch_bounds__(kSolverThreads) k_alm_post(const __grid_constant__ Solver S, Scalars* sc, const __grid_constant__ StepCfg cfg, double* nforce_out) { alm_post_body(S, sc, cfg, nforce_out); }

// update_quantities (ImplicitEulerIntegrator.cpp:13-25 or ImplicitNewmark.cpp:16-30)
// + write-back (IPCSolver.cpp:1168-1195).
__device__ __forceinline__ void update_state_body(const StepCfg& cfg, const double* x, const double* xprev, const double* vprev, const double* xhat, const double* aprev, double* pos, double* quat, double* vel, double* omega, double* lacc, double* aacc, Scalars* sc, const int* da, const int* db, const Drv* dprm, const double* dfilt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const double dt = sc->dt;
    if (i < cfg.N) {
        double vn[6], an[6];
        if (cfg.newmark) {
            const double den = (cfg.beta * dt) * dt;
            for (int k = 0; k < 6; ++k) an[k] = (x[6 * i + k] - xhat[6 * i + k]) / den;
            for (int k = 0; k < 6; ++k)
                vn[k] = vprev[6 * i + k] + dt * ((1.0 - cfg.gamma) * aprev[6 * i + k] + cfg.gamma * an[k]);
        } else {
            for (int k = 0; k < 6; ++k) vn[k] = (x[6 * i + k] - xprev[6 * i + k]) / dt;
            for (int k = 0; k < 6; ++k) an[k] = (vn[k] - vprev[6 * i + k]) / dt;
        }
        for (int k = 0; k < 3; ++k) {
            lacc[3 * i + k] = an[k]; aacc[3 * i + k] = an[3 + k];
            vel[3 * i + k] = vn[k]; omega[3 * i + k] = vn[3 + k];
            pos[3 * i + k] = x[6 * i + k];
        }
        stq(quat + 4 * i, rot_gt(ldq(quat + 4 * i), ld3(x + 6 * i + 3)));
    }
}
constexpr int kLB_update_state = 0;
__global__ void k_update_state(const __grid_constant__ StepCfg cfg, const double* x, const double* xprev, const double* vprev, const double* xhat, const double* aprev, double* pos, double* quat, double* vel, double* omega, double* lacc, double* aacc, Scalars* sc, const int* da, const int* db, const Drv* dprm, const double* dfilt) { update_state_body(cfg, x, xprev, vprev, xhat, aprev, pos, quat, vel, omega, lacc, aacc, sc, da, db, dprm, dfilt); }

// angular-velocity-drive KPIs (IPCSolver.cpp:1197-1215): only
// VelocityDriveForms are counted
__device__ __forceinline__ void drive_kpi_body(const StepCfg& cfg, const double* omega, Scalars* sc, const int* da, const int* db, const Drv* dprm, const double* dfilt, const int* dkind) {
    double max_vw = 0.0;
    int sat = 0, count = 0;
    for (int d = 0; d < cfg.D; ++d) {
        if (dkind[d] != NXD_DRIVE_ANGULAR_VELOCITY) continue;
        ++count;
        const Drv& p = dprm[d];
        const V3 oA = da[d] >= 0 ? ld3(omega + 3 * da[d]) : v3(0, 0, 0);
        const V3 oB = ld3(omega + 3 * db[d]);
        const double ve = drive_target(p, dfilt[d]) - dot(oB - oA, v3(p.ax, p.ay, p.az));
        max_vw = dmax(max_vw, fabs(ve));
        if (isfinite(p.maxT)) {
            const double tq = drive_sat(p, drive_dead(p, ve));
            if (fabs(tq) >= 0.98 * p.maxT) ++sat;
        }
    }
    sc->last_vw = max_vw;
    sc->last_tsat = count > 0 ? (double)sat / count : 0.0;
}
constexpr int kLB_drive_kpi = 0;
__global__ void k_drive_kpi(const __grid_constant__ StepCfg cfg, const double* omega, Scalars* sc, const int* da, const int* db, const Drv* dprm, const double* dfilt, const int* dkind) { drive_kpi_body(cfg, omega, sc, da, db, dprm, dfilt, dkind); }

}  // namespace nx

namespace nx {

// ---------------------------------------------------------------------------
// Form plugin interface (Dynamics/Forms/Form.h:8-21) on one CTA.
// ---------------------------------------------------------------------------
// bit masks of the forms folded into one evaluation
enum { FM_INERTIA = 1, FM_GRAVITY = 2, FM_JOINTS = 4, FM_DRIVES = 8, FM_BARRIER = 16, FM_FRICTION = 32 };

__device__ int form_mask(int form, const Solver& S) {
    switch (form) {
        case NXD_FORM_INERTIA: return FM_INERTIA;
        case NXD_FORM_GRAVITY: return FM_GRAVITY;
        case NXD_FORM_CONSTRAINT: return FM_JOINTS;
        case NXD_FORM_BARRIER: return FM_BARRIER;
        case NXD_FORM_FRICTION: return FM_FRICTION;
        case NXD_FORM_DRIVES: return FM_DRIVES;
        default: return 0;
    }
}

// what: 0 value, 1 gradient, 2 hessian block list
__global__ void __launch_bounds__(kSolverThreads) k_form_eval(Solver S, Scalars* sc, int form, int what, const double* x,
                                                              double* out, int* row_ptr, int* col_idx, double* vals,
                                                              long long cap, long long* nnzb) {
    __shared__ unsigned long long sh_keys[kMaxIncidence];
    __shared__ int sh_scan[32];
    NX_BLOCK_RED(R);
    const int N = S.N;
    const int C = sc->n_contacts;
    const double s = sc->scale;
    if (what == 0 && (form == NXD_FORM_TOTAL || form == NXD_FORM_CONTACT)) {
        const double v = energy_total(S, x, s, C, form == NXD_FORM_CONTACT, R);
        if (threadIdx.x == 0) out[0] = v;
        return;
    }
    eval_poses(S, x);
    __syncthreads();
    for (int j = threadIdx.x; j < S.J; j += blockDim.x) joint_eval(S, j, x, what > 0);
    for (int c = threadIdx.x; c < C; c += blockDim.x) {
        barrier_eval(S, c, x);
        friction_eval(S, c, x, what > 0);
    }
    for (int d = threadIdx.x; d < S.D; d += blockDim.x) drive_eval(S, d, x, what == 0 ? 0 : (what == 1 ? 1 : 2));
    __syncthreads();
    if (what == 0) {
        double v = 0.0;
        if (form == NXD_FORM_INERTIA) v = R.sum(N, [&](int i) { return inertia_value(S, i, x); });
        else if (form == NXD_FORM_GRAVITY) v = R.sum(N, [&](int i) { return gravity_value(S, i, x); });
        else if (form == NXD_FORM_CONSTRAINT) v = R.sum(S.J, [&](int j) { return S.jE[j]; });
        else if (form == NXD_FORM_BARRIER) v = R.sum(C, [&](int c) { return S.bE[c]; });
        else if (form == NXD_FORM_FRICTION) v = R.sum(C, [&](int c) { return S.fE[c]; });
        else if (form == NXD_FORM_DRIVES) v = R.sum(S.D, [&](int d) { return S.dE[d]; });
        if (threadIdx.x == 0) out[0] = v;
        return;
    }
    build_contact_incidence(S, C, sh_keys);
    if (what == 1) {
        if (form == NXD_FORM_TOTAL || form == NXD_FORM_CONTACT) {
            gather_gradient(S, x, s, C);
            __syncthreads();
            const double* src = form == NXD_FORM_TOTAL ? S.g : S.cg;
            for (int k = threadIdx.x; k < 6 * N; k += blockDim.x) out[k] = src[k];
            return;
        }
        const int m = form_mask(form, S);
        const double dh = sc->bdhat;
        const int nnf = sc->nnf;
        for (int i = threadIdx.x; i < N; i += blockDim.x) {
            double g[6] = {0, 0, 0, 0, 0, 0};
            if (m & FM_INERTIA) {
                const V3 gp = S.mass[i] * (xs3(x, 6 * i) - xs3(S.xhat, 6 * i));
                const V3 gr = mat_vec(S.inertia + 9 * i, xs3(x, 6 * i + 3) - xs3(S.xhat, 6 * i + 3));
                g[0] = gp.x; g[1] = gp.y; g[2] = gp.z; g[3] = gr.x; g[4] = gr.y; g[5] = gr.z;
            }
            if (m & FM_GRAVITY) {
                const V3 f = -S.mass[i] * v3(0.0, -9.81, 0.0);
                g[0] = f.x; g[1] = f.y; g[2] = f.z;
            }
            if (m & FM_JOINTS)
                for (int q = S.jinc_off[i]; q < S.jinc_off[i + 1]; ++q) {
                    const int j = S.jinc[q] >> 1, side = S.jinc[q] & 1;
                    const int dim = joint_dim(S.jtype[j]);
                    for (int k = 0; k < 6; ++k) {
                        double a = 0.0;
                        for (int r = 0; r < dim; ++r) a += S.jJ[72 * j + 12 * r + 6 * side + k] * S.jF[6 * j + r];
                        g[k] += a;
                    }
                }
            if (m & FM_DRIVES)
                for (int q = S.dinc_off[i]; q < S.dinc_off[i + 1]; ++q) {
                    const int d = S.dinc[q] >> 1, side = S.dinc[q] & 1;
                    for (int k = 0; k < 6; ++k) {
                        double c = 0.0;
                        const int sg = drive_grad_term(S, d, side, k, c);
                        if (sg > 0) g[k] += c;
                        else if (sg < 0) g[k] -= c;
                    }
                }
            for (int q = S.cinc_off[i]; q < S.cinc_off[i + 1]; ++q) {
                const int c = S.cinc[q] >> 1, side = S.cinc[q] & 1;
                if ((m & FM_BARRIER) && S.bD[c] < dh) {
                    const V3 n = ld3(S.contacts[c].normal);
                    const V3 contrib = side == 0 ? (-S.bGP[c]) * n : S.bGP[c] * n;
                    g[0] += contrib.x; g[1] += contrib.y; g[2] += contrib.z;
                }
                if ((m & FM_FRICTION) && c < nnf && S.nforce[c] > 0) {
                    const double* Jx = (side == 0 ? S.fJA : S.fJB) + 18 * c;
                    const V3 fg = ld3(S.fFG + 3 * c);
                    for (int k = 0; k < 6; ++k) g[k] += Jx[k] * fg.x + Jx[6 + k] * fg.y + Jx[12 + k] * fg.z;
                }
            }
            for (int k = 0; k < 6; ++k) out[6 * i + k] = g[k];
        }
        return;
    }
    // Hessian block list: row i holds its summed diagonal block, then one block
    // per coupling item incident to i (item order); like Eigen's
    // setFromTriplets the consumer sums duplicates.
    gather_diag_hessian(S, s, C);
    __syncthreads();
    const bool total = form == NXD_FORM_TOTAL;
    if (!total) {
        if (threadIdx.x == 0) *nnzb = -1;   // only the total Hessian is exported
        return;
    }
    const int n_items = S.J + S.D + 2 * C;
    for (int i = threadIdx.x; i <= N; i += blockDim.x) row_ptr[i] = i < N ? 1 : 0;
    __syncthreads();
    for (int it = threadIdx.x; it < n_items; it += blockDim.x) {
        if (!item_active(S, it)) continue;
        int a, b;
        item_bodies(S, it, a, b);
        if (a == b) continue;
        atomicAdd(&row_ptr[a], 1);
        atomicAdd(&row_ptr[b], 1);
    }
    __syncthreads();
    {
        int* const arr[1] = {row_ptr};
        block_scan_excl<1>(arr, N, sh_scan);
    }
    __syncthreads();
    const int nblocks = row_ptr[N];
    if (threadIdx.x == 0) *nnzb = nblocks;
    if (nblocks > cap) return;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        int pos = row_ptr[i];
        col_idx[pos] = i;
        for (int k = 0; k < 36; ++k) vals[36LL * pos + k] = S.Hd[36 * i + k];
        ++pos;
        for (int it = 0; it < n_items; ++it) {
            if (!item_active(S, it)) continue;
            int a, b;
            item_bodies(S, it, a, b);
            if (a == b || (a != i && b != i)) continue;
            const int other = a == i ? b : a;
            double blk[36];
            for (int k = 0; k < 36; ++k) blk[k] = 0.0;
            add_coupling_block(S, it, i, other, s, blk);
            col_idx[pos] = other;
            for (int k = 0; k < 36; ++k) vals[36LL * pos + k] = blk[k];
            ++pos;
        }
    }
}

// DistanceBarrierForm::computeNormalForces at x for the installed contacts
__global__ void k_normal_forces(Solver S, Scalars* sc, const double* x, double* out, int n) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= min(n, sc->n_contacts)) return;
    const double d = contact_distance(S.contacts[c], x);
    out[c] = (d < sc->bdhat && d > 0.0) ? fabs(barrier_gradient(d, sc->bdhat, sc->bkappa)) : 0.0;
}

// install form state (contacts are copied by the host)
__global__ void k_set_form_state(StepCfg cfg, Scalars* sc, int n, int nnf, double dt, const double* pos, const double* quat,
                                 double* pos0, double* quat0, int* dhas_prev) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < cfg.N) {
        for (int k = 0; k < 3; ++k) pos0[3 * i + k] = pos[3 * i + k];
        for (int k = 0; k < 4; ++k) quat0[4 * i + k] = quat[4 * i + k];
    }
    if (i < cfg.D) dhas_prev[i] = 0;
    if (i == 0) {
        sc->n_contacts = n;
        sc->nnf = nnf;
        sc->dt = dt;
        sc->scale = cfg.newmark ? (cfg.beta * dt) * dt : dt * dt;
        sc->friction_mu = cfg.friction_coeff;
        sc->bdhat = dmax(1e-9, sc->dhat);
        sc->bkappa = dmax(0.0, sc->kappa);
        sc->barrier_form = 1;
        sc->barrier_in_forms = cfg.enable_adaptive ? 1 : 0;
        sc->friction_form = (cfg.enable_friction && cfg.friction_coeff > 0.0) ? 1 : 0;
    }
}

}  // namespace nx
