/*
 * nxd.h — C ABI of the B200 contact step for NexDynIPC-style rigid-body IPC.
 *
 * Every entry point takes plain pointers and sizes; no CUDA or torch types
 * appear in a signature.  Each function names the reference interface it
 * replaces (paths are relative to the NexDynIPC project root).
 *
 * Conventions
 *  - Bodies are addressed by world index (position in World::bodies).  The
 *    reference maps RigidBody::id -> world index through hash maps
 *    (nexdynipc/src/Dynamics/IPCSolver.cpp:401-405); descriptors carry the ids
 *    so joints and candidates can be expressed in the reference's id space.
 *  - The optimisation vector x has 6 entries per body, [p_x p_y p_z th_x th_y
 *    th_z], th an incremental rotation vector applied as exp(th)*q_ref
 *    (IPCSolver.cpp:839-857, JointPrimitives.h:11-19).
 *  - Quaternions are stored (w, x, y, z).
 *  - All arithmetic is IEEE FP64; indices are int32.
 *  - A context owns every device buffer it uses.  Pointers passed in are host
 *    pointers unless a function says otherwise.
 */
#ifndef NXD_H
#define NXD_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (per call).  The reference signals failures only through
 * booleans (NewtonSolver::minimize, LinearSolver::info); these codes add the
 * cases a device implementation can hit. */
typedef enum nxd_status {
    NXD_OK = 0,
    NXD_NOT_CONVERGED = 1,     /* Newton hit its iteration cap            */
    NXD_LS_FAILED = 2,         /* line search returned alpha = 0          */
    NXD_FACTOR_FAILED = 3,     /* zero pivot in the LDL^T factorisation   */
    NXD_CAPACITY = 4,          /* a fixed-size device buffer overflowed   */
    NXD_NAN = 5,               /* non-finite state detected               */
    NXD_TIMEOUT = 6,           /* a bounded device loop hit its limit     */
    NXD_INVALID_ARGUMENT = 7,
    NXD_CUDA_ERROR = 8,
    NXD_NO_DEVICE = 9
} nxd_status;

/* Joint kinds, in the reference's class names. */
enum {
    NXD_JOINT_HINGE = 0,        /* HingeJoint       (Joints/HingeJoint.cpp)       */
    NXD_JOINT_FIXED = 1,        /* FixedJoint       (Joints/FixedJoint.cpp)       */
    NXD_JOINT_SPHERICAL = 2,    /* SphericalJoint   (Joints/SphericalJoint.cpp)   */
    NXD_JOINT_ANGLE_LIMIT = 3,  /* AngleLimitJoint  (Joints/AngleLimitJoint.cpp)  */
    NXD_JOINT_PRISMATIC = 4,    /* PrismaticJoint   (Joints/PrismaticJoint.cpp)   */
    NXD_JOINT_CYLINDRICAL = 5,  /* CylindricalJoint (Joints/CylindricalJoint.cpp) */
    NXD_JOINT_DISTANCE_LIMIT = 6 /* DistanceLimitJoint (Joints/DistanceLimitJoint.cpp) */
};
#define NXD_JOINT_PARAMS 16

/* Per-joint parameter layout inside nxd_scene_desc.joint_params (16 doubles):
 *   hinge:       anchorA[3] anchorB[3] axisA[3] axisB[3]      (HingeJoint ctor)
 *   fixed:       target_position[3] target_orientation[4] (w,x,y,z) (FixedJoint ctor)
 *   spherical:   anchorA[3] anchorB[3]                        (SphericalJoint ctor)
 *   angle limit: axis[3] min_angle_rad max_angle_rad          (AngleLimitJoint ctor)
 *   prismatic, cylindrical: anchorA[3] anchorB[3] axisA[3] axisB[3] (ctors)
 *   distance limit: min_distance max_distance                 (DistanceLimitJoint ctor)
 */

/* Control forms of World::forms, in load order (src/Control). */
enum {
    NXD_DRIVE_ANGULAR_VELOCITY = 0, /* VelocityDriveForm        (VelocityDriveForm.cpp)       */
    NXD_DRIVE_LINEAR_VELOCITY = 1,  /* LinearVelocityDriveForm  (LinearVelocityDriveForm.cpp) */
    NXD_DRIVE_POSITION = 2,         /* PositionDriveForm        (PositionDriveForm.cpp)       */
    NXD_DRIVE_FORCE = 3,            /* ForceDriveForm           (ForceDriveForm.cpp)          */
    NXD_DRIVE_DAMPED_SPRING = 4     /* DampedSpringForm         (DampedSpringForm.cpp)        */
};
#define NXD_DRIVE_PARAMS 8
/* Per-drive parameter layout inside nxd_scene_desc.drive_params (8 doubles):
 *   angular velocity: axis[3] kv v_target max_torque(<=0: unlimited) delay_radps delay_tau_s
 *   linear velocity:  axis[3] kv v_target max_force(<=0: unlimited)  delay_mps   delay_tau_s
 *   position:         axis[3] kp target_position max_force(<=0: unlimited) deadzone_m 0
 *   force:            force_world[3] torque_world[3] 0 0   (body_b is the body, body_a -1)
 *   damped spring:    rest_length stiffness damping 0 0 0 0 0
 * Axes are normalised at creation, as the constructors do.  body_a may be -1
 * (world) for the angular, linear and position drives; the spring needs two
 * distinct bodies. */

/* Solver settings: IPCSolver setters (Dynamics/IPCSolver.h:34-79) and
 * NewtonSolver::Options (Math/NewtonSolver.h:58-64). */
typedef struct nxd_settings {
    double dhat;                     /* setContactDistanceThreshold            */
    double contact_stiffness;        /* setContactStiffness (>0 to apply)      */
    int32_t enable_adaptive_barrier; /* enableAdaptiveBarrier                  */
    int32_t enable_ccd;              /* enableCCD                              */
    double ccd_safety_factor;        /* setCCDSafetyFactor                     */
    int32_t enable_friction;         /* enableFriction                         */
    int32_t alm_max_iters;           /* setALMMaxIters                         */
    double friction_coeff;           /* setFrictionCoefficient                 */
    double alm_constraint_tol;       /* setALMConstraintTolerance              */
    double alm_dual_tol;             /* setALMDualTolerance                    */
    double alm_contact_tol;          /* setALMContactTolerance                 */
    double alm_hardening_trigger;    /* setALMHardeningTrigger                 */
    double alm_hardening_ratio;      /* setALMHardeningRatio                   */
    int32_t newton_max_iters;        /* Options::max_iterations                */
    int32_t ls_max_iters;            /* BacktrackingLineSearch::max_iter       */
    double newton_tol;               /* Options::tolerance                     */
    double ls_c1;                    /* Options::line_search_c1                */
    double ls_rho;                   /* Options::line_search_rho               */
    int32_t integrator;              /* NXD_INTEGRATOR_* (setIntegrator)       */
    int32_t reserved0;
    double newmark_beta;             /* ImplicitNewmark(beta, gamma)           */
    double newmark_gamma;
} nxd_settings;

/* Time integrators (TimeIntegration/ImplicitTimeIntegrator.cpp:15-33):
 * implicit Euler (the IPCSolver default) and Newmark (the Simulation
 * default, beta 0.25, gamma 0.5). */
enum { NXD_INTEGRATOR_IMPLICIT_EULER = 0, NXD_INTEGRATOR_IMPLICIT_NEWMARK = 1 };

/* Fill an nxd_settings with the reference's defaults
 * (IPCSolver.h:97-119, NewtonSolver.h:58-64, LineSearch.h:36-38). */
void nxd_default_settings(nxd_settings* s);

/* A World: bodies, triangle meshes, joints and velocity drives
 * (Dynamics/World.h:11-17, Dynamics/RigidBody.h:11-38). */
typedef struct nxd_scene_desc {
    int32_t n_bodies;
    const int32_t* body_ids;             /* [n]   RigidBody::id                   */
    const double* position;              /* [n*3]                                 */
    const double* orientation;           /* [n*4] (w,x,y,z)                       */
    const double* velocity;              /* [n*3]                                 */
    const double* angular_velocity;      /* [n*3]                                 */
    const double* linear_acceleration;   /* [n*3] or NULL (zero)                  */
    const double* angular_acceleration;  /* [n*3] or NULL (zero)                  */
    const double* mass;                  /* [n]                                   */
    const double* inertia_body;          /* [n*9] row-major, body frame           */
    const int32_t* vertex_offset;        /* [n+1] prefix offsets into vertices    */
    const double* vertices;              /* [nv*3] local coordinates (MeshShape)  */
    const int32_t* face_offset;          /* [n+1] prefix offsets into faces       */
    const int32_t* faces;                /* [nf*3] body-local vertex indices      */
    int32_t n_joints;                    /* World::joints, in order               */
    const int32_t* joint_type;           /* [n_joints] NXD_JOINT_*                */
    const int32_t* joint_body_a;         /* [n_joints] body id (fixed: the body)  */
    const int32_t* joint_body_b;         /* [n_joints] body id (fixed: -1)        */
    const double* joint_params;          /* [n_joints*16]                         */
    const double* joint_stiffness;       /* [n_joints] ALM penalty mu             */
    int32_t n_drives;                    /* control forms of World::forms, load order */
    const int32_t* drive_body_a;         /* [n_drives] body id or -1 (world)      */
    const int32_t* drive_body_b;         /* [n_drives] body id                    */
    const double* drive_params;          /* [n_drives*8]                          */
    nxd_settings settings;
    /* IPCSolver::addAllowedContactPair (IPCSolver.cpp:275-289): when
     * n_contact_pairs > 0 only these body pairs make contacts, and a pair's
     * friction >= 0 overrides the friction coefficient in the per-step mean
     * over the active contacts (IPCSolver.cpp:891-911). */
    int32_t n_contact_pairs;
    const int32_t* contact_pair_bodies;  /* [n_contact_pairs*2] body ids         */
    const double* contact_pair_friction; /* [n_contact_pairs] (< 0: none) or NULL */
    const int32_t* drive_kind;           /* [n_drives] NXD_DRIVE_* or NULL (all angular velocity) */
} nxd_scene_desc;

/* Body state as written back by IPCSolver::step (IPCSolver.cpp:1174-1195). */
typedef struct nxd_state {
    double* position;              /* [n*3] */
    double* orientation;           /* [n*4] (w,x,y,z) */
    double* velocity;              /* [n*3] */
    double* angular_velocity;      /* [n*3] */
    double* linear_acceleration;   /* [n*3] */
    double* angular_acceleration;  /* [n*3] */
} nxd_state;

/* ContactPair (Dynamics/Forms/FrictionForm.h:13-22), reordered for alignment. */
typedef struct nxd_contact {
    double point[3];
    double normal[3];
    double distance;
    int32_t body_a;          /* world index */
    int32_t body_b;          /* world index */
    int32_t primitive_type;  /* 0 vertex-face or vertex-vertex, 1 edge-edge */
    int32_t primitive_a;
    int32_t primitive_b;
    int32_t pad_;
} nxd_contact;

/* ContactCandidateSet (Physics/Contact/ContactAssembler.h:12-55).  Buffers are
 * caller-owned int32 arrays; *_cap give their capacity in records; the call
 * always writes the full counts, and fails with NXD_CAPACITY if a buffer was
 * too small (records past the capacity are not written).  Any pointer may be
 * NULL to query counts only. */
typedef struct nxd_candidates {
    int32_t* vv; int64_t vv_cap; int64_t vv_count;  /* 4 ints: body0 body1 v0 v1            */
    int32_t* ev; int64_t ev_cap; int64_t ev_count;  /* 5 ints: ebody vbody e_v0 e_v1 v        */
    int32_t* ee; int64_t ee_cap; int64_t ee_count;  /* 6 ints: body0 body1 e0v0 e0v1 e1v0 e1v1 */
    int32_t* fv; int64_t fv_cap; int64_t fv_count;  /* 4 ints: fbody vbody face vertex        */
} nxd_candidates;

/* Per-step diagnostics: IPCSolver's last-step KPI getters
 * (IPCSolver.h:82-90) plus device-side counters. */
typedef struct nxd_diagnostics {
    double kappa;                    /* AdaptiveBarrier::currentStiffness       */
    double dhat;                     /* AdaptiveBarrier::currentDhat            */
    double actual_dt;                /* computeMaxStep result                   */
    double last_dual_residual;
    double last_contact_residual;
    double last_max_constraint_violation;
    double last_angular_velocity_error;
    double last_torque_saturation_ratio;
    double scene_min_distance;       /* last computeSceneMinDistance (exact when < 1e-6) */
    int32_t alm_iterations;          /* ALM iterations run in the last step     */
    int32_t newton_iterations;       /* Newton iterations summed over ALM       */
    int32_t newton_converged;        /* last Newton call's return value         */
    int32_t n_body_pairs;            /* candidate body pairs (activation dhat)  */
    int32_t n_contacts;              /* contacts after the last detection       */
    int32_t n_contacts_raw;          /* before the 2000-contact cap             */
    int32_t status;                  /* sticky nxd_status of device loops       */
    int32_t line_search_failures;    /* Newton calls that ended with alpha = 0  */
} nxd_diagnostics;

/* Form selectors for nxd_form_* (SimulationProblem, IPCSolver.cpp:137-262). */
enum {
    NXD_FORM_INERTIA = 0,     /* InertiaForm                     */
    NXD_FORM_GRAVITY = 1,     /* GravityForm (unscaled)          */
    NXD_FORM_CONSTRAINT = 2,  /* ConstraintForm over all joints  */
    NXD_FORM_BARRIER = 3,     /* DistanceBarrierForm (unscaled)  */
    NXD_FORM_FRICTION = 4,    /* FrictionForm (unscaled)         */
    NXD_FORM_DRIVES = 5,      /* sum of the control forms        */
    NXD_FORM_TOTAL = 6,       /* SimulationProblem::computeValue / computeGradient */
    NXD_FORM_CONTACT = 7      /* SimulationProblem::computeContactValue / Gradient */
};

typedef struct nxd_ctx nxd_ctx;

/* World + IPCSolver construction (App/Simulation.cpp:14-58 configuration
 * part).  Uploads the scene; afterwards no call allocates device memory
 * except when a capacity has to grow (documented per call). */
nxd_status nxd_create(const nxd_scene_desc* desc, nxd_ctx** out);
void nxd_destroy(nxd_ctx* ctx);

/* Bind the context to a CUDA stream (a cudaStream_t passed as void*). */
nxd_status nxd_set_stream(nxd_ctx* ctx, void* stream);

/* IPCSolver::step(World&, double dt) (Dynamics/IPCSolver.cpp:808-1231). */
nxd_status nxd_step(nxd_ctx* ctx, double dt);

/* Read / overwrite body state (host pointers). */
nxd_status nxd_get_state(nxd_ctx* ctx, const nxd_state* out);
nxd_status nxd_set_state(nxd_ctx* ctx, const nxd_state* in);
nxd_status nxd_get_diagnostics(nxd_ctx* ctx, nxd_diagnostics* out);
/* ALM multipliers and stiffness per joint (Joint::lambda_, Joint::mu_),
 * lambda as 6 doubles per joint (unused rows zero). */
nxd_status nxd_get_joint_state(nxd_ctx* ctx, double* lambda6, double* stiffness);

/* ContactAssembler::detectBodyPairs (ContactAssembler.cpp:156-178) on the
 * current poses.  pairs: [cap*2] world indices, in the reference's order. */
nxd_status nxd_body_pairs(nxd_ctx* ctx, double inflation_radius,
                          int32_t* pairs, int64_t cap, int64_t* count);

/* ContactAssembler::buildCandidateSet (ContactAssembler.cpp:214-343) on the
 * current poses. */
nxd_status nxd_build_candidates(nxd_ctx* ctx, double activation_distance,
                                nxd_candidates* out);

/* IPCSolver::detectContacts (IPCSolver.cpp:394-580) when x == NULL, else
 * IPCSolver::detectContactsAtState(world, x) (IPCSolver.cpp:582-806), over
 * the candidate set of the current poses with the context's current dhat. */
nxd_status nxd_detect_contacts(nxd_ctx* ctx, const double* x,
                               nxd_contact* out, int32_t cap, int32_t* count);

/* computeSceneMinDistance (Physics/Contact/AdaptiveBarrier.h:130-162).  The
 * value equals the reference's whenever the reference's is below 1e-6 (the
 * only use, AdaptiveBarrier::updateStiffness, compares it with 1e-9);
 * otherwise the call returns a value >= 1e-6 or +inf. */
nxd_status nxd_scene_min_distance(nxd_ctx* ctx, double* out);

/* IPCSolver::computeMaxStep (IPCSolver.cpp:355-392) with
 * CCDSystem::computeEarliestTOI (Physics/Contact/CCD/CCD.h:22-82). */
nxd_status nxd_max_step(nxd_ctx* ctx, double dt, double* out_dt);

/* Form plugin interface (Dynamics/Forms/Form.h:8-21) evaluated at x against
 * the contacts / normal forces / predictive state installed below.
 * value: energy; gradient: overwrites grad[6n]; hessian (NXD_FORM_TOTAL):
 * 6x6 blocks in BSR layout with caller buffers (row_ptr[n+1], col_idx[cap],
 * vals[cap*36] row-major blocks).  Like the reference's triplet list
 * (Form::hessian appends triplets that Eigen's setFromTriplets sums), a row
 * may repeat a column: its summed diagonal block comes first, then one block
 * per coupling term (joint, active barrier contact, friction contact) in term
 * order; the consumer sums duplicates.  *nnzb receives the block count
 * (NXD_CAPACITY when it exceeds cap). */
nxd_status nxd_form_value(nxd_ctx* ctx, int32_t form, const double* x, double* out);
nxd_status nxd_form_gradient(nxd_ctx* ctx, int32_t form, const double* x, double* grad);
nxd_status nxd_form_hessian_bsr(nxd_ctx* ctx, int32_t form, const double* x,
                                int32_t* row_ptr, int32_t* col_idx, double* vals,
                                int64_t cap, int64_t* nnzb);

/* SimulationProblem's three calls in one: computeValue, computeGradient and
 * computeHessian of the total energy at x (the NXD_FORM_TOTAL value,
 * gradient and BSR Hessian above; stateful drives see the value call, then
 * the gradient call, then the Hessian call). */
nxd_status nxd_eval_all(nxd_ctx* ctx, const double* x, double* energy, double* grad,
                        int32_t* row_ptr, int32_t* col_idx, double* vals, int64_t cap, int64_t* nnzb);

/* A 6x6-block sparse matrix over the context's bodies (host pointers), in the
 * layout nxd_form_hessian_bsr writes: repeated (row, col) blocks are summed in
 * storage order, as setFromTriplets sums duplicate triplets. */
typedef struct nxd_bsr {
    int32_t n_rows;             /* block rows: the context's body count */
    int64_t nnzb;               /* blocks */
    const int32_t* row_ptr;     /* [n_rows+1] */
    const int32_t* col_idx;     /* [nnzb] */
    const double* vals;         /* [nnzb*36] row-major blocks */
} nxd_bsr;

typedef struct nxd_solve_stats {
    int32_t components;         /* connected block components of 2+ bodies */
    int32_t singletons;         /* bodies coupled to no other */
    int32_t largest_component;  /* bodies in the largest component */
    int32_t factor_failed;      /* 1: an exactly zero pivot (LinearSolver::info() false) */
} nxd_solve_stats;

/* LinearSolver::analyzePattern + factorize + solve (Math/LinearSolver.cpp:11-39):
 * x = H^-1 b by block LDL^T per connected component, members ordered by
 * (coupled bodies, index), reading each block of the lower triangle in that
 * order as stored (SimplicialLDLT's UpLo = Lower).  b and x: [6 n] host
 * arrays.  NXD_FACTOR_FAILED on a zero pivot; stats may be NULL. */
nxd_status nxd_linear_solve(nxd_ctx* ctx, const nxd_bsr* H, const double* b, double* x, nxd_solve_stats* stats);

/* Block-Jacobi preconditioned conjugate gradients on a 6x6-block BSR matrix
 * (an iterative alternative to nxd_linear_solve for large systems, where a
 * direct factorisation of one big component fills in): x0 = 0, stop at
 * |r| <= tol |b| or after max_iter iterations (NXD_NOT_CONVERGED).  The
 * matrix must be symmetric positive definite (NXD_FACTOR_FAILED when a
 * diagonal block or p.Ap says otherwise); the iteration reads its upper
 * block triangle only (the diagonal blocks' upper entries and the blocks
 * with column > row; duplicates summed), as LAPACK's uplo = 'U' solvers do,
 * so the block pattern must be symmetric (NXD_INVALID_ARGUMENT otherwise).
 * H->n_rows may differ from the context's body count: only the context's
 * device and stream are used.
 * The whole iteration is one cooperative kernel; stats->kernel_ms is its
 * device time. */
typedef struct nxd_pcg_stats {
    int32_t iterations;
    int32_t status;
    double relative_residual;   /* |r| / |b| at exit */
    double kernel_ms;           /* device time of the iteration kernel */
    int32_t grid;               /* CTAs of the cooperative launch */
    int32_t threads;            /* threads per CTA */
} nxd_pcg_stats;
nxd_status nxd_pcg_solve(nxd_ctx* ctx, const nxd_bsr* H, const double* b, double* x, double tol, int32_t max_iter,
                         nxd_pcg_stats* stats);

/* DistanceBarrierForm::updateContacts + FrictionForm::updateContactPoints +
 * FrictionForm::updateNormalForces (normal_forces may be NULL: none) and
 * InertiaForm::setPredictiveState (x_hat may be NULL: keep). */
nxd_status nxd_set_form_state(nxd_ctx* ctx, const nxd_contact* contacts, int32_t n,
                              const double* normal_forces, const double* x_hat,
                              double dt);

/* DistanceBarrierForm::computeNormalForces (DistanceBarrierForm.cpp:70-86). */
nxd_status nxd_normal_forces(nxd_ctx* ctx, const double* x, double* out, int32_t n);

/* Device-side timing by kernel family, for measurement.  Every launch is
 * counted; with profiling enabled each launch is bracketed by CUDA events on
 * the context's stream.  nxd_profile(ctx, enable, ms, launches) synchronises,
 * writes the accumulated milliseconds and launch counts since the previous
 * call (arrays of NXD_PROF_FAMILIES, either may be NULL), resets them and
 * switches event timing on (enable = 1) or off (0). */
enum {
    NXD_PROF_ASSEMBLY = 0,      /* body boxes, world vertices, poses        */
    NXD_PROF_BROAD = 1,         /* body-pair broad phase                    */
    NXD_PROF_TOPK = 2,          /* top-32 primitive selection               */
    NXD_PROF_NARROW = 3,        /* narrow phase (count + ordered write)     */
    NXD_PROF_MIN_DISTANCE = 4,  /* scene minimum distance                   */
    NXD_PROF_NEWTON = 5,        /* Newton solve (one CTA per scene)         */
    NXD_PROF_ALM_POST = 6,      /* ALM convergence / normal forces          */
    NXD_PROF_SCAN = 7,          /* prefix sums                              */
    NXD_PROF_OTHER = 8,
    NXD_PROF_FAMILIES = 9
};
nxd_status nxd_profile(nxd_ctx* ctx, int32_t enable, double* ms, int64_t* launches);

/* Batched form: independent scenes (each an IPCSolver::step of its own World,
 * IPCSolver.cpp:808) stepped together.  nxd_batch_step records each scene's
 * step sequence once per set of dts; scenes whose sequences match form a
 * group, and each group's step runs as one CUDA graph of batched launches,
 * one launch per kernel for all its scenes (the Newton solve is one CTA per
 * scene).  Each scene's result equals nxd_step on its own context.
 * nxd_batch_step returns without synchronising; get_state synchronises.
 * nxd_batch_groups reports the number of groups; nxd_batch_set_stream makes
 * the batch issue its work on a caller's cudaStream_t (after synchronising
 * the previous one).  Neither has a reference counterpart.
 * The narrow-phase kernels (whose work per scene, the body-pair count, is
 * known only on the device) run in a queue form: a persistent grid of
 * ctas_per_sm CTAs per SM pulls (scene, chunk of body pairs) items from a
 * device counter.  nxd_batch_set_queue_ctas sets that grid for one kernel
 * (NXD_QUEUE_NARROW_ROWS / NXD_QUEUE_NARROW_EMIT; 1..64, default 4); the
 * results do not depend on it, only the time; the groups are rebuilt at the
 * next step. */
typedef struct nxd_batch nxd_batch;
nxd_status nxd_batch_create(const nxd_scene_desc* descs, int32_t n_scenes, nxd_batch** out);
void nxd_batch_destroy(nxd_batch* b);
nxd_status nxd_batch_step(nxd_batch* b, const double* dts);
nxd_status nxd_batch_get_state(nxd_batch* b, int32_t scene, const nxd_state* out);
nxd_status nxd_batch_get_diagnostics(nxd_batch* b, int32_t scene, nxd_diagnostics* out);
int32_t nxd_batch_groups(nxd_batch* b);
nxd_status nxd_batch_set_stream(nxd_batch* b, void* stream);
enum { NXD_QUEUE_NARROW_ROWS = 0, NXD_QUEUE_NARROW_EMIT = 1 };
nxd_status nxd_batch_set_queue_ctas(nxd_batch* b, int32_t kernel, int32_t ctas_per_sm);
/* n_steps nxd_batch_step calls timed on the batch's stream by CUDA events
 * (synchronises); used by the autotuner of the queue grids. */
nxd_status nxd_batch_timed_steps(nxd_batch* b, const double* dts, int32_t n_steps, double* ms);
/* The current device's SM count and name (the autotuner's cache key). */
nxd_status nxd_device_info(int32_t* sm_count, char* name, int32_t name_len);

/* Primitive-level contact model (full IPC).  No counterpart in the
 * reference, which only has the body-COM barrier (its design notes plan
 * this replacement: documents/2026.02.28, rigid-ipc replacement plan).
 * Primitives are numbered over bodies in world order: vertices, faces and
 * the unique edges of each body's mesh (as in nxd_build_candidates).
 * x is the 6N optimisation vector (NULL: the current poses).  Calls
 * synchronise the context's stream and return host results; device
 * buffers grow on demand.
 *
 * nxd_ipc_candidates: point-triangle pairs (vertex, face) and edge-edge
 * pairs (edge i < edge j) of different bodies whose boxes overlap, the
 * primitive box inflated by `inflation` (swept over x -> x + dx when dx is
 * given); LBVH over Morton codes.  Sorted by (first, second). */
nxd_status nxd_ipc_candidates(nxd_ctx* ctx, const double* x, const double* dx, double inflation,
                              int32_t* pt, int64_t pt_cap, int32_t* ee, int64_t ee_cap,
                              int64_t* n_pt, int64_t* n_ee);
/* nxd_ipc_barrier: the barrier form over the candidates at x (boxes
 * inflated by dhat), in the Form interface's three parts (Form.h:8-21):
 * energy sum_pairs b(d^2), b(s) = -kappa (s - dhat^2)^2 ln(s / dhat^2); the
 * gradient over the 6N DOFs (overwritten); the Hessian with each pair's
 * 12x12 block projected to PSD, chained to the two bodies' DOFs through
 * [I, -[R r]x], as BSR (row_ptr[N+1], col_idx[nnzb], vals[nnzb*36]
 * row-major).  *nnzb gets the block count (NXD_CAPACITY if > cap_blocks). */
nxd_status nxd_ipc_barrier(nxd_ctx* ctx, const double* x, double dhat, double kappa, double* energy,
                           double* grad, int32_t* row_ptr, int32_t* col_idx, double* vals,
                           int64_t cap_blocks, int64_t* nnzb, int64_t* n_pairs, int64_t* n_active);
/* nxd_ipc_max_step: the line-search bound OptimizationProblem::maxStep
 * (Math/NewtonSolver.h:42) for the step x -> x + dx: the smallest additive-CCD
 * time of impact in [0, 1] over the pairs whose swept boxes overlap, each
 * pair keeping eta of its initial distance.  The points move rigidly with
 * their bodies along the iterates x + t dx (rotation vectors interpolated,
 * so the pose at t is the one a line search evaluates at alpha = t); the
 * swept boxes (here and in nxd_ipc_candidates with dx) are padded by each
 * body's |dtheta| r_max / 2 so that they contain the rotation arcs. */
nxd_status nxd_ipc_max_step(nxd_ctx* ctx, const double* x, const double* dx, double eta, double* alpha,
                            int64_t* n_pairs);

/* Full-IPC time step: the primitive-level model above inside a Newton step.
 * x_tilde and the inertia, gravity, joint and control forms are nxd_step's
 * (joints with their current multipliers, no ALM update); the
 * primitive-pair barrier replaces the COM-distance contact forms.  Newton
 * starts from the step-start configuration and stops at |g|_inf < tol or at
 * a Newton step with |dx|_inf < tol * dt (IPC's velocity test); Armijo
 * backtracking (settings.ls_c1, ls_rho) starts from min(1, CCD bound);
 * candidates are rebuilt at every iterate and trial point; each system is
 * solved by nxd_linear_solve's factorisation or by nxd_pcg_solve's PCG
 * (linear_solver); the state is written back as nxd_step does.
 * Friction (mu > 0): the reference's smoothed friction potential
 * (FrictionPotential, Friction.cpp:5-61; D = mu lam (sqrt(|u|^2 + eps^2) -
 * eps)) on every pair active at a lag state, u the tangential displacement
 * of the pair's closest points since the step start; the pairs, their
 * normal forces lam = -db/dd, normals and closest-point weights frozen at
 * the step start, then re-frozen at each pass's solution for
 * friction_iters passes in all (the reference's lagged friction,
 * IPCSolver.cpp:1112-1130). */
typedef struct nxd_ipc_params {
    double dhat;                /* barrier activation distance               */
    double kappa;               /* barrier stiffness                         */
    double eta;                 /* CCD: kept fraction of each pair's gap     */
    double newton_tol;          /* |g|_inf                                   */
    int32_t newton_max_iters;
    int32_t ls_max_iters;
    int32_t linear_solver;      /* 0: component LDL^T (nxd_linear_solve),
                                   1: block-Jacobi PCG (nxd_pcg_solve)       */
    int32_t pcg_max_iter;
    double pcg_tol;             /* |r| / |b|                                 */
    double mu;                  /* friction coefficient (0: no friction)     */
    double friction_eps;        /* eps of the smoothed norm (m)              */
    int32_t friction_iters;     /* lagging passes (>= 1 when mu > 0)         */
    int32_t pad;
} nxd_ipc_params;
typedef struct nxd_ipc_stats {
    int32_t newton_iterations;
    int32_t converged;
    int32_t line_search_failed;
    int32_t solve_failed;
    double last_alpha_max;      /* the last CCD bound                        */
    double energy;              /* total energy at the last accepted iterate */
    int64_t n_pairs;            /* candidate pairs at the last iterate       */
    int64_t n_active;           /* pairs within dhat                         */
    int64_t pcg_iterations;     /* PCG iterations over the step              */
    int64_t n_friction;         /* frozen friction pairs of the last pass    */
} nxd_ipc_stats;
nxd_status nxd_ipc_step(nxd_ctx* ctx, double dt, const nxd_ipc_params* p, nxd_ipc_stats* stats);

/* Adjoint of one full-IPC time step (nxd_ipc_step, implicit Euler) by the
 * implicit function theorem.  No counterpart in the reference (its
 * differentiable-physics plan, documents/2026.02.21/可微物理实现方案.md, is
 * not implemented); it serves the parameter-identification workflow of
 * tools/compare_with_reference.py:85-165.  The step solves G(x; z) = 0
 * for x = (p, theta) per body; at its converged iterate x_star (6N: the new
 * positions and angular_velocity * dt), for x_bar = dL/dx_star:
 *   K^T lambda = x_bar,  K = dG/dx (exact, unprojected, symmetric),
 * and the input adjoints -(dG/dz)^T lambda: phat_bar = m lambda_p (the
 * predicted position p0 + dt v0), thetahat_bar = I^T lambda_theta (the
 * predicted rotation dt w0), phi_bar (left rotations of the step-start
 * orientations, tangent 3-vectors), mass_bar, inertia_bar (3x3 per body,
 * row-major), joint_mu_bar (fixed joints' stiffness).  `start` is the step's
 * input state (host arrays); the context is left at that state.  Supported:
 * bodies, fixed joints (FixedJoint), no control forms, implicit Euler,
 * N <= 128 bodies (dense K, one CTA); else NXD_INVALID_ARGUMENT.
 * Friction (p->mu > 0) with one lagging pass (friction_iters = 1): the pairs
 * frozen at the step start enter K, and, through their frozen normal
 * forces, normals, closest-point weights and displacement origin, the
 * step-start positions (p0_bar, added to what reaches p0 through the
 * predicted position) and orientations (phi_bar); friction_mu_bar is the
 * coefficient's adjoint.  More lagging passes: NXD_INVALID_ARGUMENT.
 * NXD_FACTOR_FAILED if K is singular.  Output pointers are host arrays and
 * may be NULL. */
typedef struct nxd_ipc_adjoint_out {
    double* lambda;             /* [6N] */
    double* phat_bar;           /* [3N] */
    double* thetahat_bar;       /* [3N] */
    double* phi_bar;            /* [3N] */
    double* mass_bar;           /* [N]  */
    double* inertia_bar;        /* [9N] */
    double* joint_mu_bar;       /* [J]  */
    int32_t* n_active;          /* active pairs at x_star (may be NULL) */
    double* p0_bar;             /* [3N] step-start positions through the frozen
                                   friction pairs (mu > 0; may be NULL)     */
    double* friction_mu_bar;    /* [1]  the friction coefficient (may be NULL) */
} nxd_ipc_adjoint_out;
nxd_status nxd_ipc_adjoint(nxd_ctx* ctx, double dt, const nxd_ipc_params* p, const nxd_state* start,
                           const double* x_star, const double* x_bar, const nxd_ipc_adjoint_out* out);

/* Body-pair broad phase for callers that cannot allocate device memory.
 * No counterpart in the reference.  Callers that manage every device byte
 * themselves (a host engine's memory pool, a hard memory cap, a real-time
 * loop that forbids allocator calls) pass device buffers they own:
 * position [n*3], orientation [n*4] (w,x,y,z), local_box [n*6] (local AABB
 * min xyz, max xyz, i.e. MeshShape::computeAABB) and pairs [cap*2].  A body
 * without a mesh (no vertices or no faces) takes part in no pair, as in
 * nxd_body_pairs: pass its local box empty, min > max on some axis (e.g.
 * min = (1,1,1), max = (-1,-1,-1)); a NaN bound counts as empty too.  The
 * result equals nxd_body_pairs on the same poses (reference order); *count
 * (host) gets the pair count, NXD_CAPACITY if it exceeds cap (the first cap
 * pairs are written, nothing past pairs[2*cap)).
 * The call allocates nothing: its scratch (world boxes, per-body counts and
 * offsets, about 0.9 MB) is a fixed array in the library that every GPU which
 * loads it holds until exit, so n is limited to NXD_NOALLOC_MAX_BODIES
 * (larger n -> NXD_INVALID_ARGUMENT).  The first call on a device looks up
 * that array's device address; make it before any stream capture.  All calls
 * share the one array: calls that overlap on the GPU (different streams)
 * race.  The call synchronises `stream` (a cudaStream_t, may be NULL) before
 * returning the count.  The looked-up address is kept for the life of the
 * process: a cudaDeviceReset (or any teardown of the device's primary
 * context) after the first call is not supported. */
#define NXD_NOALLOC_MAX_BODIES 16384
nxd_status nxd_body_pairs_noalloc(const double* position, const double* orientation, const double* local_box,
                                  int32_t n, double inflation_radius, int32_t* pairs, int64_t cap,
                                  int64_t* count, void* stream);

/* Failure-detection hook, no counterpart in the reference (its Newton solve
 * has no waits and no failure report).  spin_limit > 0 bounds every grid-
 * barrier wait of the Newton solve to that many polls (at most 2^20);
 * hold_last_cta != 0 (needs spin_limit > 0) makes the solve's last CTA keep
 * away from its first barrier until the others have given up (at most
 * 64 x spin_limit polls), so their waits run out: the step then reports
 * NXD_TIMEOUT in nxd_diagnostics.status and every CTA returns.  Both switch
 * the solve to the global-memory barrier, whose waits are bounded (the
 * cluster form waits in hardware).  nxd_debug_grid_wait(ctx, 0, 0) restores
 * the normal solve and clears the sticky status; the context stays usable
 * (set the state again before stepping on).  Synchronises the context's
 * stream. */
nxd_status nxd_debug_grid_wait(nxd_ctx* ctx, uint32_t spin_limit, int32_t hold_last_cta);

/* FP64 fused multiply-add throughput of the current device, in TFLOP/s
 * (best of five timed launches of independent DFMA chains on every SM; *ms
 * gets that launch's time, may be NULL).  A measurement helper for the FP64
 * rooflines, with no counterpart in the reference; it allocates and frees a
 * few KB and synchronises `stream`. */
nxd_status nxd_fp64_peak(void* stream, double* tflops, double* ms);

/* Library version string. */
const char* nxd_version(void);

#ifdef __cplusplus
}
#endif

#endif /* NXD_H */
