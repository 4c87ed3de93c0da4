// nxd.cu — host side of the B200 contact step: the context that owns every
// device buffer, the per-step kernel sequence of IPCSolver::step, and the C
// ABI declared in include/nxd.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <new>
#include <unordered_set>
#include <vector>

#include "../../include/nxd.h"
#include "step.cuh"
#include "batch.cuh"
#include "ipc.cuh"
#include "adjoint.cuh"
#include "pcg.cuh"

using namespace nx;

namespace {

#define NXD_CUDA(call)                                                   \
    do {                                                                 \
        cudaError_t e_ = (call);                                         \
        if (e_ != cudaSuccess) {                                         \
            std::fprintf(stderr, "nxd: %s failed: %s\n", #call, cudaGetErrorString(e_)); \
            return NXD_CUDA_ERROR;                                       \
        }                                                                \
    } while (0)

struct DevArena {
    std::vector<void*> ptrs;
    bool ok = true;
    template <typename T>
    T* alloc(size_t n) {
        void* p = nullptr;
        if (n == 0) n = 1;
        if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) { ok = false; return nullptr; }
        cudaMemset(p, 0, n * sizeof(T));
        ptrs.push_back(p);
        return static_cast<T*>(p);
    }
    template <typename T>
    T* upload(const T* h, size_t n) {
        T* d = alloc<T>(n);
        if (d && h && n) cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice);
        return d;
    }
    void release() {
        for (void* p : ptrs) cudaFree(p);
        ptrs.clear();
    }
};


int grid_for(long long n, int block, int max_blocks = 1 << 16) {
    long long g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > max_blocks) g = max_blocks;
    return (int)g;
}

}  // namespace

struct nxd_ctx {
    DevArena mem;
    // launch accounting (always) and per-family device timing (when enabled)
    long long launches[NXD_PROF_FAMILIES] = {};
    bool prof = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev[NXD_PROF_FAMILIES];
    std::vector<cudaEvent_t> pool;
    cudaStream_t stream = nullptr;
    int dev = 0, n_sm = 148;
    int newton_grid = 1;   // co-resident CTAs of k_newton (power of two)
    bool newton_cluster = false;   // k_newton's CTAs launched as one thread-block cluster
    int N = 0, nv = 0, nf = 0, ne = 0, J = 0, D = 0;
    int max_prims = 0;
    int max_verts = 0;
    int pair_cap = 0;
    nxd_settings s{};
    std::vector<int> h_body_ids;
    std::vector<int> h_jtype;
    std::vector<int> h_voff, h_foff, h_eoff;
    // static device data
    Geo geo{};
    int *voff, *foff, *eoff, *faces, *edges, *vbody, *has_mesh, *body_ids;
    double *verts, *lmin, *lmax, *md_tol, *max_md_tol;
    double *mass, *inertia;
    int *jtype, *ja, *jb, *jinc_off, *jinc;
    double *jparams, *jmu, *jlam;
    int *da, *db, *dinc_off, *dinc, *dfinit, *dhas_prev;
    Drv* dprm;
    int* dkind;
    double* dDir;
    double *dfilt, *dprevA, *dprevB;
    // state
    double *pos, *quat, *vel, *omega, *lacc, *aacc;
    // per step
    double *boxes, *wv, *wvx, *pose_p, *pose_q;
    double *x, *xhat, *xprev, *vprev, *aprev, *pos0, *quat0;
    int *pair_cnt, *pair_off, *pairs, *md_pairs;
    int *topk, *topn;
    int *nfv, *nee, *nvv, *nev, *off_fv, *off_ee, *off_vv, *off_ev;
    int *hit_cnt, *hit_off;          // narrow-phase hits per pair: FV | EE halves, and their prefixes
    unsigned* hmask;                 // narrow-phase column hit masks, kMaskWords per pair
    ContactRec *contacts, *contacts_tmp;
    double* sort_key;
    int* sort_idx;
    int *sort_g, *sort_l;       // G / L position lists of the contact sort's partitions
    SortRange* sort_small;      // ranges the contact sort finishes one warp each
    double* nforce;
    Scalars* sc;
    int* i_scratch;   // small int scalars for scans
    // solver scratch
    Solver S{};
    int cand_stride = 0;
    // allowed contact pairs (sorted keys) and their friction overrides
    unsigned long long* allowed_keys = nullptr;
    double* allowed_mu = nullptr;
    int n_allowed = 0;
    bool has_mu_override = false;
    // when set, launches are recorded here (batched replay) instead of issued
    std::vector<LaunchRec>* rec = nullptr;
    // primitive-level (full IPC) model state, created on first use
    struct IpcState* ipc = nullptr;
    // nxd_step as a CUDA graph, captured per dt on a private stream
    cudaStream_t cap_stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    double graph_dt = 0.0;
    bool graph_off = false;
    long long graph_launches[NXD_PROF_FAMILIES] = {};
};

namespace {

cudaEvent_t prof_event(nxd_ctx* c) {
    if (!c->pool.empty()) { cudaEvent_t e = c->pool.back(); c->pool.pop_back(); return e; }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}
struct ProfScope {
    nxd_ctx* c; int fam; cudaEvent_t a = nullptr;
    ProfScope(nxd_ctx* c_, int f) : c(c_), fam(f) {
        c->launches[fam] += 1;
        if (c->prof) { a = prof_event(c); cudaEventRecord(a, c->stream); }
    }
    ~ProfScope() {
        if (c->prof) { cudaEvent_t b = prof_event(c); cudaEventRecord(b, c->stream); c->ev[fam].push_back({a, b}); }
    }
};
#define NXD_LAUNCH(ctx, fam, ...) do { ProfScope ps_(ctx, fam); __VA_ARGS__; } while (0)
// Launch of a step kernel k_<name> (body <name>_body): issued on the
// context's stream, or recorded for a batched replay.
#define NXD_K(ctx, fam, name, grid, block, smem, ...)                                                     \
    do {                                                                                                \
        if ((ctx)->rec) {                                                                               \
            record_into<&name##_body, kLB_##name>(*(ctx)->rec, fam, (decltype(&name##_body))nullptr,    \
                                                   dim3(grid), dim3(block), (size_t)(smem), __VA_ARGS__); \
        } else {                                                                                        \
            ProfScope ps_(ctx, fam);                                                                    \
            k_##name<<<grid, block, smem, (ctx)->stream>>>(__VA_ARGS__);                                \
        }                                                                                               \
    } while (0)

// A launch of a narrow-phase kernel k_<name> (body <name>_body with a
// trailing block index and count, item counter <name>_items): plain, or
// recorded in the queue form for a batched replay (queue kind qk).
#define NXD_KQ(ctx, fam, qk, name, grid, block, smem, ...)                                                      \
    do {                                                                                                      \
        if ((ctx)->rec) {                                                                                     \
            record_queue_into<&name##_body, &name##_items, kLB_##name>(*(ctx)->rec, fam, qk, &name##_items,   \
                                                                       dim3(grid), dim3(block), (size_t)(smem), \
                                                                       __VA_ARGS__);                          \
        } else {                                                                                              \
            ProfScope ps_(ctx, fam);                                                                          \
            k_##name<<<grid, block, smem, (ctx)->stream>>>(__VA_ARGS__);                                      \
        }                                                                                                     \
    } while (0)
enum { kQueueNarrowRows = 0, kQueueNarrowEmit = 1, kQueueKinds = 2 };

void configure_newton_launch(nxd_ctx* c);

void fill_solver(nxd_ctx* c) {
    Solver& S = c->S;
    const int N = c->N, J = c->J, D = c->D, C = kMaxRawContacts;
    DevArena& m = c->mem;
    S.N = N; S.J = J; S.D = D; S.Cmax = C;
    S.mass = c->mass; S.inertia = c->inertia;
    S.pos0 = c->pos0; S.quat0 = c->quat0;
    S.x = c->x; S.xhat = c->xhat;
    S.jtype = c->jtype; S.ja = c->ja; S.jb = c->jb; S.jparams = c->jparams; S.jmu = c->jmu; S.jlam = c->jlam;
    S.jinc_off = c->jinc_off; S.jinc = c->jinc;
    S.da = c->da; S.db = c->db; S.dprm = c->dprm; S.dprevA = c->dprevA; S.dprevB = c->dprevB;
    S.dkind = c->dkind; S.dDir = c->dDir; S.bvel = c->vel;
    S.dhas_prev = c->dhas_prev; S.dfilt = c->dfilt; S.dinc_off = c->dinc_off; S.dinc = c->dinc;
    S.contacts = c->contacts; S.ncontacts_ptr = &c->sc->n_contacts;
    S.nforce = c->nforce; S.nnf_ptr = &c->sc->nnf;
    S.cinc_off = m.alloc<int>(N + 1); S.cinc = m.alloc<int>(2 * C);
    S.heavy = m.alloc<int>(N); S.heavy_list = m.alloc<int>(N); S.n_heavy = m.alloc<int>(1);
    S.dt_ptr = &c->sc->dt; S.scale_ptr = &c->sc->scale; S.bdhat_ptr = &c->sc->bdhat; S.bkappa_ptr = &c->sc->bkappa;
    S.barrier_in_forms_ptr = &c->sc->barrier_in_forms; S.friction_form_ptr = &c->sc->friction_form;
    S.friction_mu_ptr = &c->sc->friction_mu; S.friction_eps = 1e-8;
    S.newton_max_iters = c->s.newton_max_iters; S.ls_max_iters = c->s.ls_max_iters;
    S.newton_tol = c->s.newton_tol; S.ls_c1 = c->s.ls_c1; S.ls_rho = c->s.ls_rho;
    S.alm_constraint_tol = c->s.alm_constraint_tol; S.alm_hardening_trigger = c->s.alm_hardening_trigger;
    S.alm_hardening_ratio = c->s.alm_hardening_ratio;
    S.g = m.alloc<double>(6 * N); S.cg = m.alloc<double>(6 * N); S.dx = m.alloc<double>(6 * N);
    S.xt = m.alloc<double>(6 * N);
    S.qj = m.alloc<double>(4 * N); S.qg = m.alloc<double>(4 * N);
    S.jC = m.alloc<double>(6 * J); S.jF = m.alloc<double>(6 * J); S.jJ = m.alloc<double>(72 * J);
    S.jE = m.alloc<double>(J); S.jact = m.alloc<int>(J);
    S.bD = m.alloc<double>(C); S.bGP = m.alloc<double>(C); S.bHP = m.alloc<double>(C); S.bE = m.alloc<double>(C);
    S.fFG = m.alloc<double>(3 * C); S.fHF = m.alloc<double>(9 * C); S.fJA = m.alloc<double>(18 * C);
    S.fJB = m.alloc<double>(18 * C); S.fE = m.alloc<double>(C);
    S.dE = m.alloc<double>(D); S.dG = m.alloc<double>(D); S.dH = m.alloc<double>(D);
    S.Hd = m.alloc<double>(36 * N);
    S.parent = m.alloc<int>(N + 1); S.comp = m.alloc<int>(N);
    S.mcnt = m.alloc<int>(N + 1); S.icnt = m.alloc<int>(N + 1); S.rflag = m.alloc<int>(N + 1);
    S.comp_root = m.alloc<int>(N + 1); S.n_comp = m.alloc<int>(1); S.comp_next = m.alloc<int>(1);
    S.members = m.alloc<int>(N); S.items = m.alloc<int>(J + D + 2 * kMaxContacts); S.local = m.alloc<int>(N + 1);
    // per-component structure masks (3 k ceil(k/32) words + lists) and factors
    // (36 (k + nnz(L)) + 6k doubles, nnz(L) <= k(k-1)/2): room for the whole
    // scene as one dense component, the factor pool capped at 768 MB
    const long long kk = std::min<long long>(N, kMaxComponentBodies);
    const long long mwords = 3LL * kk * ((kk + 31) / 32) + 16LL * N + 4LL * (J + D + 2 * kMaxContacts) + 4096;
    S.mpool = m.alloc<unsigned>(mwords); S.mpool_cap = mwords; S.mpool_off = m.alloc<long long>(1);
    const long long pool_doubles = std::min<long long>(96LL << 20, 18LL * N * N + 64LL * N + 4096);
    S.pool = m.alloc<double>(pool_doubles); S.pool_cap = pool_doubles; S.pool_off = m.alloc<long long>(1);
    S.alm_done = &c->sc->alm_done; S.status = &c->sc->status; S.newton_iters = &c->sc->newton_iters;
    S.converged = &c->sc->converged; S.ls_fail = &c->sc->ls_fail;
    S.alm_mcv = m.alloc<double>(1); S.alm_dual = m.alloc<double>(1);
    S.solve_fail = m.alloc<int>(1);
    S.iact = m.alloc<int>(J + D + 2 * kMaxContacts);
    S.ext_n = -1; S.ext_row = nullptr; S.ext_col = nullptr; S.ext_vals = nullptr;
    S.bar_count = m.alloc<unsigned>(2); S.bar_abort = (int*)(S.bar_count + 1);
    S.spin_limit = 0; S.dbg_hold = 0;
    S.gpart = m.alloc<double>(2 * kRedMaxQ * kMaxNewtonGrid);
    // one CTA of kNewtonThreads per 512 DOFs, a power of two no larger than
    // what the device keeps co-resident
    S.slab_bytes = kNewtonSlabBytes;
    cudaFuncSetAttribute(k_newton, cudaFuncAttributeMaxDynamicSharedMemorySize, kNewtonDynSmem);
    cudaFuncSetAttribute(k_linear_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, kNewtonDynSmem);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_newton, kNewtonThreads, kNewtonDynSmem);
    const int coresident = std::max(1, per_sm * c->n_sm);
    int g = 1;
    while (g < kMaxNewtonGrid && g * 2 <= coresident && (long long)g * kNewtonThreads < 6LL * N) g *= 2;
    c->newton_grid = g;
    configure_newton_launch(c);
}

// Up to 16 CTAs of k_newton run as one thread-block cluster (hardware grid
// barrier) when the device can place such a cluster; NXD_NEWTON_BARRIER=global
// keeps the cooperative launch with the global-memory barrier.
void configure_newton_launch(nxd_ctx* c) {
    const int g = c->newton_grid;
    c->newton_cluster = false;
    const char* nb = std::getenv("NXD_NEWTON_BARRIER");
    if (g > 1 && g <= 16 && !(nb && std::strcmp(nb, "global") == 0)) {
        cudaFuncSetAttribute(k_newton, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(g); cfg.blockDim = dim3(kNewtonThreads); cfg.dynamicSmemBytes = kNewtonDynSmem;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = g; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
        cfg.attrs = at; cfg.numAttrs = 1;
        int ncl = 0;
        if (cudaOccupancyMaxActiveClusters(&ncl, (const void*)k_newton, &cfg) == cudaSuccess && ncl >= 1)
            c->newton_cluster = true;
        cudaGetLastError();
    }
}

StepCfg step_cfg(const nxd_ctx* c) {
    StepCfg k;
    k.N = c->N; k.D = c->D;
    k.enable_adaptive = c->s.enable_adaptive_barrier;
    k.enable_friction = c->s.enable_friction;
    k.friction_coeff = c->s.friction_coeff;
    k.alm_constraint_tol = c->s.alm_constraint_tol;
    k.alm_dual_tol = c->s.alm_dual_tol;
    k.alm_contact_tol = c->s.alm_contact_tol;
    k.newmark = c->s.integrator == NXD_INTEGRATOR_IMPLICIT_NEWMARK ? 1 : 0;
    k.beta = c->s.newmark_beta;
    k.gamma = c->s.newmark_gamma;
    return k;
}

// one ALM iteration's Newton solve: one CTA (a plain launch; the grid
// barrier degenerates to __syncthreads), or barrier counters zeroed and a
// cooperative launch of k_newton on c->newton_grid co-resident CTAs
void launch_newton(nxd_ctx* c) {
    if (c->rec || c->newton_grid == 1) {
        NXD_K(c, NXD_PROF_NEWTON, newton, (1), (kNewtonThreads), (kNewtonDynSmem), c->S);
        return;
    }
    ProfScope ps_(c, NXD_PROF_NEWTON);
    if (c->newton_cluster) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(c->newton_grid); cfg.blockDim = dim3(kNewtonThreads);
        cfg.dynamicSmemBytes = kNewtonDynSmem; cfg.stream = c->stream;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = c->newton_grid; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
        cfg.attrs = at; cfg.numAttrs = 1;
        cudaLaunchKernelEx(&cfg, k_newton, c->S);
        return;
    }
    cudaMemsetAsync(c->S.bar_count, 0, 2 * sizeof(unsigned), c->stream);
    void* args[] = {(void*)&c->S};
    cudaLaunchCooperativeKernel((const void*)k_newton, dim3(c->newton_grid), dim3(kNewtonThreads), args, kNewtonDynSmem, c->stream);
}

// ContactAssembler::build + world vertices at the current poses
void launch_assembly(nxd_ctx* c) {
    NXD_K(c, NXD_PROF_ASSEMBLY, body_boxes, (grid_for(c->N, 128)), (128), (0), c->geo, c->pos, c->quat, c->boxes);
    NXD_K(c, NXD_PROF_ASSEMBLY, world_vertices, (grid_for(c->nv, 256)), (256), (0), c->geo, c->nv, c->vbody, c->pos, c->quat, c->wv);
}

// pair list (count / scan / write) with query q into out, count -> *count_dev
void launch_pairs(nxd_ctx* c, const PairQuery& q, int* out, int* count_dev, const int* gate) {
    const int blocks = grid_for((long long)c->N * 32, 256);
    NXD_K(c, NXD_PROF_BROAD, pairs, (blocks), (256), (0), c->geo, q, c->boxes, c->pair_cnt, nullptr, nullptr, 0, gate);
    NXD_K(c, NXD_PROF_SCAN, scan, (1), (1024), (0), c->pair_cnt, c->pair_off, c->N, count_dev, gate, nullptr, nullptr);
    NXD_K(c, NXD_PROF_BROAD, pairs, (blocks), (256), (0), c->geo, q, c->boxes, nullptr, c->pair_off, out, c->pair_cap, gate);
}

// CTAs of a grid-stride loop over the pair list: no more than the pair
// capacity or N(N-1)/2 pairs can need a warp, so a small world (a batch
// replays hundreds of them in one launch) launches only the CTAs it can use
int pair_grid(const nxd_ctx* c, int warps_per_pair_item, int items_per_pair, int warps_per_block, int max_blocks) {
    const long long maxp = std::min<long long>(c->pair_cap, (long long)c->N * (c->N - 1) / 2);
    const long long warps = maxp * items_per_pair * warps_per_pair_item;
    const long long need = (warps + warps_per_block - 1) / warps_per_block;
    return (int)std::max<long long>(1, std::min<long long>(max_blocks, need));
}

size_t topk_smem(const nxd_ctx* c, int warps) {
    return (size_t)warps * topk_warp_bytes(c->max_prims, c->max_verts);
}

// buildCandidateSet with activation distance = *dhat (device) -> pairs, topk, item offsets
void launch_candidates(nxd_ctx* c, const double* act_ptr, double act_val) {
    PairQuery q{1, act_ptr, act_val, 1.0, 1.0};
    launch_pairs(c, q, c->pairs, &c->sc->n_pairs, nullptr);
    int warps = 8;
    while (warps > 1 && topk_smem(c, warps) > 200 * 1024) --warps;
    NXD_K(c, NXD_PROF_TOPK, topk, (pair_grid(c, 1, 2, warps, c->n_sm * 4)), (32 * warps), (topk_smem(c, warps)), c->geo, c->pairs, &c->sc->n_pairs, c->pair_cap,
                                                                       c->boxes, c->wv, c->topk, c->topn, c->max_prims, c->max_verts);
}

}  // namespace

namespace {

// detectContacts (current poses) or detectContactsAtState(x) over the step's
// candidate set: FV then EE passes (hit counts, ordered writes), the VV
// fallback when both found nothing, then the raw cap and the 2000 cap.
// skip_if (device flag, may be null) skips the whole detection.
void launch_narrow_full(nxd_ctx* c, const double* wv, const double* pose_p, const int* skip_if) {
    NarrowIn in{c->geo, c->pairs, &c->sc->n_pairs, c->pair_cap, c->topk, c->topn, wv, pose_p, &c->sc->dhat,
                c->allowed_keys, c->n_allowed};
    const NarrowScratch ns{c->hmask, c->hit_cnt, c->hit_off};
    const int rows_blocks = pair_grid(c, 1, 1, kRowsWarps, c->n_sm * 8);
    const int emit_blocks = pair_grid(c, 1, 1, kEmitWarps, c->n_sm * 2);
    int* skip_vv = c->i_scratch;
    const int* np = &c->sc->n_pairs;
    NXD_KQ(c, NXD_PROF_NARROW, kQueueNarrowRows, narrow_rows, (rows_blocks), (32 * kRowsWarps), (0), in, 0, ns, skip_if);
    NXD_K(c, NXD_PROF_SCAN, hit_scan, (1), (1024), (0), c->hit_cnt, c->hit_off, c->pair_cap, np, 2, &c->sc->fv_hits,
                                                                      &c->sc->ee_hits, skip_if);
    NXD_KQ(c, NXD_PROF_NARROW, kQueueNarrowEmit, narrow_emit, (emit_blocks), (32 * kEmitWarps), (0), in, 0, ns,
           &c->sc->fv_hits, c->contacts, skip_if);
    NXD_K(c, NXD_PROF_OTHER, contact_totals, (1), (1), (0), c->sc, 0, skip_if, skip_vv);
    NXD_KQ(c, NXD_PROF_NARROW, kQueueNarrowRows, narrow_rows, (rows_blocks), (32 * kRowsWarps), (0), in, 1, ns, skip_vv);
    NXD_K(c, NXD_PROF_SCAN, hit_scan, (1), (1024), (0), c->hit_cnt, c->hit_off, c->pair_cap, np, 1, &c->sc->vv_hits,
                                                                      nullptr, skip_vv);
    NXD_KQ(c, NXD_PROF_NARROW, kQueueNarrowEmit, narrow_emit, (emit_blocks), (32 * kEmitWarps), (0), in, 1, ns, nullptr,
           c->contacts, skip_vv);
    NXD_K(c, NXD_PROF_OTHER, contact_totals, (1), (1), (0), c->sc, 1, skip_if, nullptr);
    NXD_K(c, NXD_PROF_OTHER, sort_contacts, (1), (1024), (sort_smem_bytes(32)), c->sc, c->contacts, c->contacts_tmp, c->sort_key,
          c->sort_idx, c->sort_g, c->sort_l, c->sort_small, skip_if);
}

}  // namespace

// A detection pass inside an ALM iteration runs only when the iteration runs
// and a contact form exists; fold both conditions into one skip flag.
__device__ __forceinline__ void alm_detect_gate_body(const Scalars* sc, int* skip) {
    *skip = (sc->alm_done || !(sc->barrier_form || sc->friction_form)) ? 1 : 0;
}
constexpr int kLB_alm_detect_gate = 0;
__global__ void k_alm_detect_gate(const Scalars* sc, int* skip) { alm_detect_gate_body(sc, skip); }
__device__ __forceinline__ void init_scalar_d_body(double* p, double v) { *p = v; }
constexpr int kLB_init_scalar_d = 0;
__global__ void k_init_scalar_d(double* p, double v) { init_scalar_d_body(p, v); }
// max(0, tol[0..n)) over one CTA (the tolerances are positive and finite, so
// the maximum does not depend on the order)
__device__ __forceinline__ void max_tol_body(const double* tol, int n, double* out) {
    NX_BLOCK_RED(R);
    double m = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) m = dmax(m, tol[i]);
    m = R.max(m);
    if (threadIdx.x == 0) *out = m;
}
constexpr int kLB_max_tol = kSolverThreads;
__global__ void __launch_bounds__(kSolverThreads) k_max_tol(const double* tol, int n, double* out) { max_tol_body(tol, n, out); }
__device__ __forceinline__ void body_md_tol_body(const Geo& g, const double* pos, double* tol) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.N) return;
    const double diag = norm(ld3(g.lmax + 3 * i) - ld3(g.lmin + 3 * i));
    tol[i] = 4e-6 * diag + 1e-9 * (1.0 + norm(ld3(pos + 3 * i)) + diag);
}
constexpr int kLB_body_md_tol = 0;
__global__ void k_body_md_tol(const __grid_constant__ Geo g, const double* pos, double* tol) { body_md_tol_body(g, pos, tol); }

namespace {

nxd_status enqueue_step(nxd_ctx* c, double dt) {
    const StepCfg cfg = step_cfg(c);
    // ContactAssembler::build + buildCandidateSet(currentDhat)
    launch_assembly(c);
    launch_candidates(c, &c->sc->dhat, 0.0);
    // adaptive barrier (IPCSolver.cpp:817-832)
    if (c->s.enable_adaptive_barrier) {
        NXD_K(c, NXD_PROF_OTHER, barrier_init, (1), (kSolverThreads), (0), cfg, c->mass, c->pos, c->sc);
        NXD_K(c, NXD_PROF_OTHER, init_scalar_d, (1), (1), (0), &c->sc->bmd, INFINITY);
        PairQuery qb{0, &c->sc->dhat, 0.0, 2.0, 0.0};
        NXD_K(c, NXD_PROF_BROAD, min_pair_distance, (grid_for((long long)c->N * 32, 256)), (256), (0), c->geo, qb, c->boxes, &c->sc->bmd);
        NXD_K(c, NXD_PROF_OTHER, body_md_tol, (grid_for(c->N, 128)), (128), (0), c->geo, c->pos, c->md_tol);
        NXD_K(c, NXD_PROF_OTHER, max_tol, (1), (kSolverThreads), (0), c->md_tol, c->N, c->max_md_tol);
        NXD_K(c, NXD_PROF_OTHER, md_gate, (1), (1), (0), c->sc, c->max_md_tol);
        PairQuery qm{2, &c->sc->md_radius, 0.0, 1.0, 0.0};
        launch_pairs(c, qm, c->md_pairs, &c->sc->n_md_pairs, &c->sc->md_gate);
        NXD_K(c, NXD_PROF_MIN_DISTANCE, min_distance, (pair_grid(c, 1, 1, 8, c->n_sm * 4)), (256), (0), c->geo, c->md_pairs, &c->sc->n_md_pairs, c->pair_cap, c->boxes, c->wv,
                                                    &c->sc->md, &c->sc->md_gate);
        NXD_K(c, NXD_PROF_OTHER, kappa_update, (1), (1), (0), c->sc);
    }
    // computeMaxStep: the FV root box fails the reference's domain predicate
    // before any bisection, so the earliest TOI is 1 and the step is dt.
    // integrator init, contact forms, drives
    NXD_K(c, NXD_PROF_OTHER, step_setup, (grid_for(std::max(c->N, c->D), 128)), (128), (0), cfg, dt, c->pos, c->quat, c->vel, c->omega, c->lacc, c->aacc, c->x, c->xhat, c->xprev, c->vprev, c->aprev, c->pos0,
        c->quat0, c->sc, c->dprm, c->dfilt, c->dfinit, c->dhas_prev);
    // detectContacts at the step-start poses (when a contact form is needed)
    const bool needs = c->s.enable_adaptive_barrier || (c->s.enable_friction && c->s.friction_coeff > 0.0);
    if (needs) launch_narrow_full(c, c->wv, c->pos, nullptr);
    else NXD_K(c, NXD_PROF_OTHER, contact_totals, (1), (1), (0), c->sc, 2, nullptr, nullptr);
    // the friction form's coefficient with per-pair overrides, from the
    // step-start contacts (IPCSolver.cpp:891-911)
    if (c->has_mu_override && c->s.enable_friction && c->s.friction_coeff > 0.0)
        NXD_K(c, NXD_PROF_OTHER, friction_mu, (1), (1), (0), cfg, c->sc, c->contacts, c->allowed_keys, c->allowed_mu, c->n_allowed);
    int* skip_detect = c->i_scratch + 1;
    for (int alm = 0; alm < c->s.alm_max_iters; ++alm) {
        launch_newton(c);
        NXD_K(c, NXD_PROF_OTHER, alm_detect_gate, (1), (1), (0), c->sc, skip_detect);
        NXD_K(c, NXD_PROF_ASSEMBLY, pose_at_x, (grid_for(c->N, 128)), (128), (0), c->N, c->x, c->quat, c->pose_p, c->pose_q);
        NXD_K(c, NXD_PROF_ASSEMBLY, world_vertices, (grid_for(c->nv, 256)), (256), (0), c->geo, c->nv, c->vbody, c->pose_p, c->pose_q, c->wvx);
        launch_narrow_full(c, c->wvx, c->pose_p, skip_detect);
        NXD_K(c, NXD_PROF_ALM_POST, alm_post, (1), (kSolverThreads), (0), c->S, c->sc, cfg, c->nforce);
    }
    NXD_K(c, NXD_PROF_OTHER, update_state, (grid_for(c->N, 128)), (128), (0), cfg, c->x, c->xprev, c->vprev, c->xhat, c->aprev, c->pos, c->quat, c->vel, c->omega,
                                                        c->lacc, c->aacc, c->sc, c->da, c->db, c->dprm, c->dfilt);
    if (c->D > 0) NXD_K(c, NXD_PROF_OTHER, drive_kpi, (1), (1), (0), cfg, c->omega, c->sc, c->da, c->db, c->dprm, c->dfilt, c->dkind);
    NXD_CUDA(cudaGetLastError());
    return NXD_OK;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
namespace {
void drop_step_graph(nxd_ctx* c);
void configure_newton_launch(nxd_ctx* c);
void release_ipc(nxd_ctx* c);
}  // namespace

extern "C" {

void nxd_default_settings(nxd_settings* s) {
    std::memset(s, 0, sizeof(*s));
    s->dhat = 1e-3;
    s->contact_stiffness = -1.0;
    s->enable_adaptive_barrier = 1;
    s->enable_ccd = 1;
    s->ccd_safety_factor = 0.8;
    s->enable_friction = 0;
    s->alm_max_iters = 10;
    s->friction_coeff = 0.0;
    s->alm_constraint_tol = 1e-4;
    s->alm_dual_tol = 1e-3;
    s->alm_contact_tol = 1e-3;
    s->alm_hardening_trigger = 2.0;
    s->alm_hardening_ratio = 2.0;
    s->newton_max_iters = 20;
    s->ls_max_iters = 20;
    s->newton_tol = 1e-6;
    s->ls_c1 = 1e-4;
    s->ls_rho = 0.5;
    s->integrator = NXD_INTEGRATOR_IMPLICIT_EULER;
    s->newmark_beta = 0.25;
    s->newmark_gamma = 0.5;
}

const char* nxd_version(void) { return "nxd-b200 0.1 (sm_100a, FP64)"; }

nxd_status nxd_create(const nxd_scene_desc* d, nxd_ctx** out) {
    if (!d || !out || d->n_bodies <= 0 || !d->position || !d->orientation || !d->mass || !d->inertia_body ||
        !d->vertex_offset || !d->face_offset)
        return NXD_INVALID_ARGUMENT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return NXD_NO_DEVICE;
    nxd_ctx* c = new (std::nothrow) nxd_ctx();
    if (!c) return NXD_INVALID_ARGUMENT;
    cudaGetDevice(&c->dev);
    cudaDeviceGetAttribute(&c->n_sm, cudaDevAttrMultiProcessorCount, c->dev);
    c->s = d->settings;
    const int N = d->n_bodies;
    c->N = N;
    c->J = d->n_joints;
    c->D = d->n_drives;
    c->h_voff.assign(d->vertex_offset, d->vertex_offset + N + 1);
    c->h_foff.assign(d->face_offset, d->face_offset + N + 1);
    c->nv = c->h_voff[N];
    c->nf = c->h_foff[N];
    c->h_body_ids.resize(N);
    for (int i = 0; i < N; ++i) c->h_body_ids[i] = d->body_ids ? d->body_ids[i] : i;
    auto idx_of = [&](int id) -> int {
        for (int i = 0; i < N; ++i) if (c->h_body_ids[i] == id) return i;
        return -1;
    };
    // static mesh topology: unique edges in first-seen order
    // (build_unique_edges, ContactAssembler.cpp:90-120), local AABBs
    // (MeshShape ctor, MeshShape.cpp:6-11), vertex -> body map
    std::vector<int> edges, eoff(N + 1, 0), vbody(c->nv), has_mesh(N, 0);
    std::vector<double> lmin(3 * N, 0.0), lmax(3 * N, 0.0);
    for (int i = 0; i < N; ++i) {
        const int v0 = c->h_voff[i], v1 = c->h_voff[i + 1], f0 = c->h_foff[i], f1 = c->h_foff[i + 1];
        for (int v = v0; v < v1; ++v) vbody[v] = i;
        eoff[i] = (int)(edges.size() / 2);
        if (v1 > v0 && f1 > f0) {
            has_mesh[i] = 1;
            for (int k = 0; k < 3; ++k) { lmin[3 * i + k] = d->vertices[3 * v0 + k]; lmax[3 * i + k] = d->vertices[3 * v0 + k]; }
            for (int v = v0; v < v1; ++v)
                for (int k = 0; k < 3; ++k) {
                    lmin[3 * i + k] = std::min(lmin[3 * i + k], d->vertices[3 * v + k]);
                    lmax[3 * i + k] = std::max(lmax[3 * i + k], d->vertices[3 * v + k]);
                }
            std::unordered_set<unsigned long long> seen;
            for (int f = f0; f < f1; ++f) {
                const int* F = d->faces + 3 * f;
                const int pr[3][2] = {{F[0], F[1]}, {F[1], F[2]}, {F[2], F[0]}};
                for (auto& e : pr) {
                    const int lo = std::min(e[0], e[1]), hi = std::max(e[0], e[1]);
                    const unsigned long long key = ((unsigned long long)(unsigned)lo << 32) | (unsigned)hi;
                    if (seen.insert(key).second) { edges.push_back(lo); edges.push_back(hi); }
                }
            }
        }
        const int nvb = v1 - v0, nfb = f1 - f0, neb = (int)(edges.size() / 2) - eoff[i];
        c->max_prims = std::max({c->max_prims, nvb, nfb, neb});
        c->max_verts = std::max(c->max_verts, nvb);
    }
    eoff[N] = (int)(edges.size() / 2);
    c->ne = eoff[N];
    c->h_eoff = eoff;
    // joints: world indices, angle-limit axis normalised (AngleLimitJoint ctor)
    std::vector<int> jtype(c->J), ja(c->J), jb(c->J);
    std::vector<double> jparams((size_t)16 * c->J), jmu(c->J), jlam((size_t)6 * c->J, 0.0);
    std::vector<std::vector<int>> jinc_l(N), dinc_l(N);
    for (int j = 0; j < c->J; ++j) {
        jtype[j] = d->joint_type[j];
        ja[j] = idx_of(d->joint_body_a[j]);
        jb[j] = jtype[j] == NXD_JOINT_FIXED ? -1 : idx_of(d->joint_body_b[j]);
        if (ja[j] < 0 || (jtype[j] != NXD_JOINT_FIXED && jb[j] < 0) || jtype[j] < 0 || jtype[j] > NXD_JOINT_DISTANCE_LIMIT) {
            c->mem.release(); delete c; return NXD_INVALID_ARGUMENT;
        }
        for (int k = 0; k < 16; ++k) jparams[16 * j + k] = d->joint_params[16 * j + k];
        if (jtype[j] == NXD_JOINT_ANGLE_LIMIT) {
            V3 a = normalized(v3(jparams[16 * j], jparams[16 * j + 1], jparams[16 * j + 2]));
            jparams[16 * j] = a.x; jparams[16 * j + 1] = a.y; jparams[16 * j + 2] = a.z;
        }
        jmu[j] = d->joint_stiffness[j];
        jinc_l[ja[j]].push_back(2 * j);
        if (jb[j] >= 0) jinc_l[jb[j]].push_back(2 * j + 1);
    }
    std::vector<int> da(c->D), db(c->D);
    std::vector<Drv> dprm(c->D);
    std::vector<double> dfilt(c->D);
    std::vector<int> dkind(c->D, NXD_DRIVE_ANGULAR_VELOCITY);
    for (int k = 0; k < c->D; ++k) {
        const int kind = d->drive_kind ? d->drive_kind[k] : NXD_DRIVE_ANGULAR_VELOCITY;
        dkind[k] = kind;
        da[k] = d->drive_body_a[k] >= 0 ? idx_of(d->drive_body_a[k]) : -1;
        db[k] = idx_of(d->drive_body_b[k]);
        // the loader's checks (SceneLoader.cpp:274-446): body_b must exist (an
        // unknown body_a is the world), a spring needs both bodies; a form
        // coupling a body to itself is refused
        const bool bad = kind < NXD_DRIVE_ANGULAR_VELOCITY || kind > NXD_DRIVE_DAMPED_SPRING || db[k] < 0 ||
                         da[k] == db[k] ||
                         (kind == NXD_DRIVE_DAMPED_SPRING && da[k] < 0) || (kind == NXD_DRIVE_FORCE && da[k] >= 0);
        if (bad) { c->mem.release(); delete c; return NXD_INVALID_ARGUMENT; }
        const double* p = d->drive_params + 8 * k;
        if (kind == NXD_DRIVE_FORCE || kind == NXD_DRIVE_DAMPED_SPRING) {
            dprm[k] = Drv{p[0], p[1], p[2], p[3], p[4], p[5], 0.0, 0.0};
        } else {
            // constructors normalise the axis; setMaxForce / setMaxTorque map
            // <= 0 to unlimited; setDelay / setDeadzone / setDelayTau clamp at 0
            const V3 ax = normalized(v3(p[0], p[1], p[2]));
            const double tau = kind == NXD_DRIVE_POSITION ? 0.0 : std::max(0.0, p[7]);
            dprm[k] = Drv{ax.x, ax.y, ax.z, p[3], p[4], p[5] <= 0.0 ? INFINITY : p[5], std::max(0.0, p[6]), tau};
        }
        dfilt[k] = p[4];
        if (da[k] >= 0) dinc_l[da[k]].push_back(2 * k);
        dinc_l[db[k]].push_back(2 * k + 1);
    }
    auto csr = [&](const std::vector<std::vector<int>>& L, std::vector<int>& off, std::vector<int>& val) {
        off.assign(N + 1, 0);
        for (int i = 0; i < N; ++i) { off[i + 1] = off[i] + (int)L[i].size(); for (int v : L[i]) val.push_back(v); }
    };
    std::vector<int> jinc_off, jinc, dinc_off, dinc;
    csr(jinc_l, jinc_off, jinc);
    csr(dinc_l, dinc_off, dinc);

    DevArena& m = c->mem;
    c->voff = m.upload(c->h_voff.data(), N + 1);
    c->foff = m.upload(c->h_foff.data(), N + 1);
    c->eoff = m.upload(eoff.data(), N + 1);
    c->verts = m.upload(d->vertices, (size_t)3 * c->nv);
    c->faces = m.upload(d->faces, (size_t)3 * c->nf);
    c->edges = m.upload(edges.data(), edges.size());
    c->vbody = m.upload(vbody.data(), vbody.size());
    c->has_mesh = m.upload(has_mesh.data(), N);
    c->body_ids = m.upload(c->h_body_ids.data(), N);
    // IPCSolver::addAllowedContactPair: keys of world-index pairs, sorted,
    // with the last non-negative friction given for a pair as its override
    if (d->n_contact_pairs > 0 && d->contact_pair_bodies) {
        std::vector<std::pair<unsigned long long, double>> kv;
        for (int q = 0; q < d->n_contact_pairs; ++q) {
            const int a = idx_of(d->contact_pair_bodies[2 * q]), b = idx_of(d->contact_pair_bodies[2 * q + 1]);
            if (a < 0 || b < 0) continue;
            const int lo = std::min(a, b), hi = std::max(a, b);
            const double f = d->contact_pair_friction ? d->contact_pair_friction[q] : -1.0;
            kv.push_back({((unsigned long long)(unsigned)lo << 32) | (unsigned)hi, f});
        }
        std::stable_sort(kv.begin(), kv.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
        std::vector<unsigned long long> keys;
        std::vector<double> mu;
        for (const auto& e : kv) {
            if (!keys.empty() && keys.back() == e.first) { if (e.second >= 0.0) mu.back() = e.second; continue; }
            keys.push_back(e.first);
            mu.push_back(e.second >= 0.0 ? e.second : -1.0);
        }
        for (double f : mu) c->has_mu_override = c->has_mu_override || f >= 0.0;
        c->n_allowed = (int)keys.size();
        c->allowed_keys = m.upload(keys.data(), keys.size());
        c->allowed_mu = m.upload(mu.data(), mu.size());
    }
    c->lmin = m.upload(lmin.data(), 3 * N);
    c->lmax = m.upload(lmax.data(), 3 * N);
    c->md_tol = m.alloc<double>(N);
    c->max_md_tol = m.alloc<double>(1);
    c->mass = m.upload(d->mass, N);
    c->inertia = m.upload(d->inertia_body, (size_t)9 * N);
    c->jtype = m.upload(jtype.data(), c->J); c->ja = m.upload(ja.data(), c->J); c->jb = m.upload(jb.data(), c->J);
    c->h_jtype.assign(jtype.begin(), jtype.end());
    c->jparams = m.upload(jparams.data(), jparams.size()); c->jmu = m.upload(jmu.data(), c->J);
    c->jlam = m.upload(jlam.data(), jlam.size());
    c->jinc_off = m.upload(jinc_off.data(), N + 1); c->jinc = m.upload(jinc.data(), jinc.size());
    c->da = m.upload(da.data(), c->D); c->db = m.upload(db.data(), c->D); c->dprm = m.upload(dprm.data(), c->D);
    c->dkind = m.upload(dkind.data(), c->D); c->dDir = m.alloc<double>(3 * c->D);
    c->dfilt = m.upload(dfilt.data(), c->D); c->dfinit = m.alloc<int>(c->D); c->dhas_prev = m.alloc<int>(c->D);
    c->dprevA = m.alloc<double>(3 * c->D); c->dprevB = m.alloc<double>(3 * c->D);
    c->dinc_off = m.upload(dinc_off.data(), N + 1); c->dinc = m.upload(dinc.data(), dinc.size());
    std::vector<double> zeros(3 * N, 0.0);
    c->pos = m.upload(d->position, 3 * N);
    c->quat = m.upload(d->orientation, 4 * N);
    c->vel = m.upload(d->velocity ? d->velocity : zeros.data(), 3 * N);
    c->omega = m.upload(d->angular_velocity ? d->angular_velocity : zeros.data(), 3 * N);
    c->lacc = m.upload(d->linear_acceleration ? d->linear_acceleration : zeros.data(), 3 * N);
    c->aacc = m.upload(d->angular_acceleration ? d->angular_acceleration : zeros.data(), 3 * N);
    c->geo = Geo{N, c->voff, c->foff, c->eoff, c->verts, c->faces, c->edges, c->lmin, c->lmax, c->has_mesh, c->md_tol};
    c->boxes = m.alloc<double>(6 * N);
    c->wv = m.alloc<double>(3 * (size_t)c->nv); c->wvx = m.alloc<double>(3 * (size_t)c->nv);
    c->pose_p = m.alloc<double>(3 * N); c->pose_q = m.alloc<double>(4 * N);
    c->x = m.alloc<double>(6 * N); c->xhat = m.alloc<double>(6 * N); c->xprev = m.alloc<double>(6 * N);
    c->vprev = m.alloc<double>(6 * N); c->aprev = m.alloc<double>(6 * N);
    c->pos0 = m.alloc<double>(3 * N); c->quat0 = m.alloc<double>(4 * N);
    c->pair_cap = std::max(4096, 16 * N);
    c->pair_cnt = m.alloc<int>(N); c->pair_off = m.alloc<int>(N);
    c->pairs = m.alloc<int>(2 * (size_t)c->pair_cap); c->md_pairs = m.alloc<int>(2 * (size_t)c->pair_cap);
    c->topk = m.alloc<int>((size_t)c->pair_cap * 6 * kTopK); c->topn = m.alloc<int>((size_t)c->pair_cap * 6);
    c->nfv = m.alloc<int>(c->pair_cap); c->nee = m.alloc<int>(c->pair_cap); c->nvv = m.alloc<int>(c->pair_cap);
    c->nev = m.alloc<int>(c->pair_cap);
    c->off_fv = m.alloc<int>(c->pair_cap); c->off_ee = m.alloc<int>(c->pair_cap); c->off_vv = m.alloc<int>(c->pair_cap);
    c->off_ev = m.alloc<int>(c->pair_cap);
    c->hit_cnt = m.alloc<int>(2 * (size_t)c->pair_cap); c->hit_off = m.alloc<int>(2 * (size_t)c->pair_cap);
    c->hmask = m.alloc<unsigned>((size_t)c->pair_cap * kMaskWords);
    c->contacts = m.alloc<ContactRec>(kMaxRawContacts);
    c->contacts_tmp = m.alloc<ContactRec>(kMaxContacts);
    c->sort_key = m.alloc<double>(kMaxRawContacts); c->sort_idx = m.alloc<int>(kMaxRawContacts);
    c->sort_g = m.alloc<int>(kMaxRawContacts + 1); c->sort_l = m.alloc<int>(kMaxRawContacts + 1);
    c->sort_small = m.alloc<SortRange>(kMaxContacts + kSortWarpRange + 64);
    c->nforce = m.alloc<double>(kMaxRawContacts);
    c->sc = m.alloc<Scalars>(1);
    c->i_scratch = m.alloc<int>(16);
    Scalars hs{};
    hs.dhat = std::max(1e-9, c->s.dhat);
    hs.kappa = c->s.contact_stiffness > 0.0 ? c->s.contact_stiffness : 0.0;
    hs.bmd = INFINITY;
    hs.md = INFINITY;
    cudaMemcpy(c->sc, &hs, sizeof(hs), cudaMemcpyHostToDevice);
    fill_solver(c);
    // top-k kernel needs opt-in shared memory above 48 KB
    cudaFuncSetAttribute(k_topk, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
    cudaFuncSetAttribute(k_sort_contacts, cudaFuncAttributeMaxDynamicSharedMemorySize, sort_smem_bytes(32));
    if (!m.ok || cudaDeviceSynchronize() != cudaSuccess) {
        m.release();
        delete c;
        return NXD_CUDA_ERROR;
    }
    *out = c;
    return NXD_OK;
}

void nxd_destroy(nxd_ctx* c) {
    if (!c) return;
    cudaDeviceSynchronize();
    for (auto& v : c->ev)
        for (auto& pr : v) { cudaEventDestroy(pr.first); cudaEventDestroy(pr.second); }
    for (cudaEvent_t e : c->pool) cudaEventDestroy(e);
    drop_step_graph(c);
    release_ipc(c);
    if (c->cap_stream) cudaStreamDestroy(c->cap_stream);
    c->mem.release();
    delete c;
}

nxd_status nxd_set_stream(nxd_ctx* c, void* stream) {
    if (!c) return NXD_INVALID_ARGUMENT;
    c->stream = static_cast<cudaStream_t>(stream);
    return NXD_OK;
}

}  // extern "C"

namespace {

void drop_step_graph(nxd_ctx* c) {
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    if (c->graph) cudaGraphDestroy(c->graph);
    c->graph_exec = nullptr;
    c->graph = nullptr;
}

// Captures enqueue_step(c, dt) into c->graph_exec; false if the capture or
// the instantiation is refused (the step then runs as direct launches).
bool capture_step(nxd_ctx* c, double dt) {
    drop_step_graph(c);
    if (!c->cap_stream && cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking) != cudaSuccess) return false;
    long long before[NXD_PROF_FAMILIES];
    std::memcpy(before, c->launches, sizeof(before));
    cudaStream_t saved = c->stream;
    c->stream = c->cap_stream;
    bool ok = cudaStreamBeginCapture(c->cap_stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
        const nxd_status st = enqueue_step(c, dt);
        const cudaError_t e = cudaStreamEndCapture(c->cap_stream, &c->graph);
        ok = st == NXD_OK && e == cudaSuccess && c->graph;
    }
    c->stream = saved;
    for (int f = 0; f < NXD_PROF_FAMILIES; ++f) {
        c->graph_launches[f] = c->launches[f] - before[f];
        c->launches[f] = before[f];
    }
    if (ok) ok = cudaGraphInstantiate(&c->graph_exec, c->graph, 0) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        drop_step_graph(c);
        return false;
    }
    c->graph_dt = dt;
    return true;
}

}  // namespace

extern "C" {

nxd_status nxd_step(nxd_ctx* c, double dt) {
    if (!c || !(dt > 0.0)) return NXD_INVALID_ARGUMENT;
    // per-family event timing needs direct launches
    if (c->prof || c->graph_off) return enqueue_step(c, dt);
    if (!c->graph_exec || c->graph_dt != dt) {
        if (!capture_step(c, dt)) {
            c->graph_off = true;
            return enqueue_step(c, dt);
        }
    }
    for (int f = 0; f < NXD_PROF_FAMILIES; ++f) c->launches[f] += c->graph_launches[f];
    NXD_CUDA(cudaGraphLaunch(c->graph_exec, c->stream));
    return NXD_OK;
}

nxd_status nxd_debug_grid_wait(nxd_ctx* c, uint32_t spin_limit, int32_t hold_last_cta) {
    if (!c || spin_limit > (1u << 20) || (hold_last_cta && spin_limit == 0)) return NXD_INVALID_ARGUMENT;
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return NXD_CUDA_ERROR;
    drop_step_graph(c);                 // the captured step holds the old settings
    c->S.spin_limit = spin_limit;
    c->S.dbg_hold = hold_last_cta ? 1 : 0;
    if (spin_limit || hold_last_cta) {
        c->newton_cluster = false;      // the hardware barrier has no bounded form
    } else {
        configure_newton_launch(c);
        // back to normal: the sticky status of the failed step is cleared
        if (cudaMemsetAsync(&c->sc->status, 0, sizeof(int), c->stream) != cudaSuccess ||
            cudaStreamSynchronize(c->stream) != cudaSuccess)
            return NXD_CUDA_ERROR;
    }
    return NXD_OK;
}

// State copies are queued on the context's stream behind the work already
// there (one copy per array, no batched-copy API), then waited for once, so
// the host buffers are free when the call returns.
nxd_status nxd_get_state(nxd_ctx* c, const nxd_state* o) {
    if (!c || !o) return NXD_INVALID_ARGUMENT;
    const size_t n3 = 3 * (size_t)c->N * sizeof(double), n4 = 4 * (size_t)c->N * sizeof(double);
    const cudaMemcpyKind k = cudaMemcpyDeviceToHost;
    if (o->position) NXD_CUDA(cudaMemcpyAsync(o->position, c->pos, n3, k, c->stream));
    if (o->orientation) NXD_CUDA(cudaMemcpyAsync(o->orientation, c->quat, n4, k, c->stream));
    if (o->velocity) NXD_CUDA(cudaMemcpyAsync(o->velocity, c->vel, n3, k, c->stream));
    if (o->angular_velocity) NXD_CUDA(cudaMemcpyAsync(o->angular_velocity, c->omega, n3, k, c->stream));
    if (o->linear_acceleration) NXD_CUDA(cudaMemcpyAsync(o->linear_acceleration, c->lacc, n3, k, c->stream));
    if (o->angular_acceleration) NXD_CUDA(cudaMemcpyAsync(o->angular_acceleration, c->aacc, n3, k, c->stream));
    NXD_CUDA(cudaStreamSynchronize(c->stream));
    return NXD_OK;
}

nxd_status nxd_set_state(nxd_ctx* c, const nxd_state* o) {
    if (!c || !o) return NXD_INVALID_ARGUMENT;
    const size_t n3 = 3 * (size_t)c->N * sizeof(double), n4 = 4 * (size_t)c->N * sizeof(double);
    const cudaMemcpyKind k = cudaMemcpyHostToDevice;
    if (o->position) NXD_CUDA(cudaMemcpyAsync(c->pos, o->position, n3, k, c->stream));
    if (o->orientation) NXD_CUDA(cudaMemcpyAsync(c->quat, o->orientation, n4, k, c->stream));
    if (o->velocity) NXD_CUDA(cudaMemcpyAsync(c->vel, o->velocity, n3, k, c->stream));
    if (o->angular_velocity) NXD_CUDA(cudaMemcpyAsync(c->omega, o->angular_velocity, n3, k, c->stream));
    if (o->linear_acceleration) NXD_CUDA(cudaMemcpyAsync(c->lacc, o->linear_acceleration, n3, k, c->stream));
    if (o->angular_acceleration) NXD_CUDA(cudaMemcpyAsync(c->aacc, o->angular_acceleration, n3, k, c->stream));
    NXD_CUDA(cudaStreamSynchronize(c->stream));
    return NXD_OK;
}

nxd_status nxd_get_diagnostics(nxd_ctx* c, nxd_diagnostics* o) {
    if (!c || !o) return NXD_INVALID_ARGUMENT;
    NXD_CUDA(cudaStreamSynchronize(c->stream));
    Scalars h;
    NXD_CUDA(cudaMemcpy(&h, c->sc, sizeof(h), cudaMemcpyDeviceToHost));
    std::memset(o, 0, sizeof(*o));
    o->kappa = h.kappa; o->dhat = h.dhat; o->actual_dt = h.dt;
    o->last_dual_residual = h.alm_dual; o->last_contact_residual = h.alm_cres;
    o->last_max_constraint_violation = h.alm_mcv;
    o->last_angular_velocity_error = h.last_vw; o->last_torque_saturation_ratio = h.last_tsat;
    o->scene_min_distance = h.md;
    o->alm_iterations = h.alm_iters; o->newton_iterations = h.newton_iters; o->newton_converged = h.converged;
    o->n_body_pairs = h.n_pairs; o->n_contacts = h.n_contacts; o->n_contacts_raw = h.n_contacts_raw;
    o->status = h.status | ((h.n_pairs > c->pair_cap || h.n_md_pairs > c->pair_cap) ? NXD_CAPACITY : 0);
    o->line_search_failures = h.ls_fail;
    return NXD_OK;
}

nxd_status nxd_get_joint_state(nxd_ctx* c, double* lambda6, double* stiffness) {
    if (!c) return NXD_INVALID_ARGUMENT;
    NXD_CUDA(cudaStreamSynchronize(c->stream));
    if (lambda6 && c->J) NXD_CUDA(cudaMemcpy(lambda6, c->jlam, 6 * (size_t)c->J * sizeof(double), cudaMemcpyDeviceToHost));
    if (stiffness && c->J) NXD_CUDA(cudaMemcpy(stiffness, c->jmu, (size_t)c->J * sizeof(double), cudaMemcpyDeviceToHost));
    return NXD_OK;
}

nxd_status nxd_body_pairs(nxd_ctx* c, double r, int32_t* pairs, int64_t cap, int64_t* count) {
    if (!c || !count) return NXD_INVALID_ARGUMENT;
    launch_assembly(c);
    PairQuery q{0, nullptr, r, 1.0, 0.0};
    launch_pairs(c, q, c->md_pairs, &c->sc->n_md_pairs, nullptr);
    NXD_CUDA(cudaStreamSynchronize(c->stream));
    int n = 0;
    NXD_CUDA(cudaMemcpy(&n, &c->sc->n_md_pairs, sizeof(int), cudaMemcpyDeviceToHost));
    *count = n;
    if (n > c->pair_cap) return NXD_CAPACITY;
    if (pairs && cap > 0)
        NXD_CUDA(cudaMemcpy(pairs, c->md_pairs, 2 * sizeof(int) * (size_t)std::min<int64_t>(n, cap), cudaMemcpyDeviceToHost));
    return n > cap && pairs ? NXD_CAPACITY : NXD_OK;
}

nxd_status nxd_build_candidates(nxd_ctx* c, double act, nxd_candidates* o) {
    if (!c || !o) return NXD_INVALID_ARGUMENT;
    launch_assembly(c);
    launch_candidates(c, nullptr, act);
    // per-pair item counts and offsets of the four candidate lists
    NXD_K(c, NXD_PROF_OTHER, item_counts, (grid_for(c->pair_cap, 256)), (256), (0), &c->sc->n_pairs, c->pair_cap, c->topn, c->nfv, c->nee,
                                                                       c->nvv, c->nev);
    const int* np = &c->sc->n_pairs;
    NXD_K(c, NXD_PROF_SCAN, scan, (1), (1024), (0), c->nfv, c->off_fv, c->pair_cap, &c->sc->fv_items, nullptr, nullptr, np);
    NXD_K(c, NXD_PROF_SCAN, scan, (1), (1024), (0), c->nee, c->off_ee, c->pair_cap, &c->sc->ee_items, nullptr, nullptr, np);
    NXD_K(c, NXD_PROF_SCAN, scan, (1), (1024), (0), c->nvv, c->off_vv, c->pair_cap, &c->sc->vv_items, nullptr, nullptr, np);
    int* tot = c->i_scratch + 4;
    NXD_K(c, NXD_PROF_SCAN, scan, (1), (1024), (0), c->nev, c->off_ev, c->pair_cap, tot, nullptr, nullptr, &c->sc->n_pairs);
    NXD_CUDA(cudaStreamSynchronize(c->stream));
    Scalars h;
    int nev_total = 0;
    NXD_CUDA(cudaMemcpy(&h, c->sc, sizeof(h), cudaMemcpyDeviceToHost));
    NXD_CUDA(cudaMemcpy(&nev_total, tot, sizeof(int), cudaMemcpyDeviceToHost));
    if (h.n_pairs > c->pair_cap) return NXD_CAPACITY;
    o->vv_count = h.vv_items; o->ev_count = nev_total; o->ee_count = h.ee_items; o->fv_count = h.fv_items;
    nxd_status st = NXD_OK;
    auto need = [&](int32_t* buf, int64_t cap, int64_t cnt) { if (buf && cnt > cap) st = NXD_CAPACITY; };
    need(o->vv, o->vv_cap, o->vv_count); need(o->ev, o->ev_cap, o->ev_count);
    need(o->ee, o->ee_cap, o->ee_count); need(o->fv, o->fv_cap, o->fv_count);
    if (!o->vv && !o->ev && !o->ee && !o->fv) return st;
    DevArena tmp;
    CandOut co{};
    co.vv = tmp.alloc<int>(4 * (size_t)std::max<int64_t>(1, o->vv_count)); co.vv_cap = o->vv_count;
    co.ev = tmp.alloc<int>(5 * (size_t)std::max<int64_t>(1, o->ev_count)); co.ev_cap = o->ev_count;
    co.ee = tmp.alloc<int>(6 * (size_t)std::max<int64_t>(1, o->ee_count)); co.ee_cap = o->ee_count;
    co.fv = tmp.alloc<int>(4 * (size_t)std::max<int64_t>(1, o->fv_count)); co.fv_cap = o->fv_count;
    if (!tmp.ok) { tmp.release(); return NXD_CUDA_ERROR; }
    NXD_LAUNCH(c, NXD_PROF_OTHER, k_materialize<<<c->n_sm * 4, 256, 0, c->stream>>>(c->geo, c->body_ids, c->pairs, &c->sc->n_pairs, c->pair_cap, c->topk,
                                                     c->topn, c->off_vv, c->off_ev, c->off_ee, c->off_fv, co););
    cudaStreamSynchronize(c->stream);
    auto back = [&](int32_t* buf, int64_t cap, const int* dev, int64_t cnt, int w) {
        if (buf && cnt > 0) cudaMemcpy(buf, dev, sizeof(int) * w * (size_t)std::min(cap, cnt), cudaMemcpyDeviceToHost);
    };
    back(o->vv, o->vv_cap, co.vv, o->vv_count, 4);
    back(o->ev, o->ev_cap, co.ev, o->ev_count, 5);
    back(o->ee, o->ee_cap, co.ee, o->ee_count, 6);
    back(o->fv, o->fv_cap, co.fv, o->fv_count, 4);
    tmp.release();
    return st;
}

nxd_status nxd_detect_contacts(nxd_ctx* c, const double* x, nxd_contact* out, int32_t cap, int32_t* count) {
    if (!c) return NXD_INVALID_ARGUMENT;
    launch_assembly(c);
    launch_candidates(c, &c->sc->dhat, 0.0);
    if (x) {
        NXD_CUDA(cudaMemcpyAsync(c->S.xt, x, 6 * (size_t)c->N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        NXD_K(c, NXD_PROF_ASSEMBLY, pose_at_x, (grid_for(c->N, 128)), (128), (0), c->N, c->S.xt, c->quat, c->pose_p, c->pose_q);
        NXD_K(c, NXD_PROF_ASSEMBLY, world_vertices, (grid_for(c->nv, 256)), (256), (0), c->geo, c->nv, c->vbody, c->pose_p, c->pose_q, c->wvx);
        launch_narrow_full(c, c->wvx, c->pose_p, nullptr);
    } else {
        launch_narrow_full(c, c->wv, c->pos, nullptr);
    }
    NXD_CUDA(cudaStreamSynchronize(c->stream));
    Scalars h;
    NXD_CUDA(cudaMemcpy(&h, c->sc, sizeof(h), cudaMemcpyDeviceToHost));
    if (count) *count = h.n_contacts;
    if (out && cap > 0)
        NXD_CUDA(cudaMemcpy(out, c->contacts, sizeof(nxd_contact) * (size_t)std::min(cap, h.n_contacts), cudaMemcpyDeviceToHost));
    return h.n_contacts > cap && out ? NXD_CAPACITY : NXD_OK;
}

nxd_status nxd_scene_min_distance(nxd_ctx* c, double* out) {
    if (!c || !out) return NXD_INVALID_ARGUMENT;
    launch_assembly(c);
    cudaStream_t st = c->stream;
    NXD_K(c, NXD_PROF_OTHER, body_md_tol, (grid_for(c->N, 128)), (128), (0), c->geo, c->pos, c->md_tol);
    NXD_K(c, NXD_PROF_OTHER, max_tol, (1), (kSolverThreads), (0), c->md_tol, c->N, c->max_md_tol);
    // force the gate open: bmd = 0
    NXD_K(c, NXD_PROF_OTHER, init_scalar_d, (1), (1), (0), &c->sc->bmd, 0.0);
    NXD_K(c, NXD_PROF_OTHER, md_gate, (1), (1), (0), c->sc, c->max_md_tol);
    PairQuery qm{2, &c->sc->md_radius, 0.0, 1.0, 0.0};
    launch_pairs(c, qm, c->md_pairs, &c->sc->n_md_pairs, &c->sc->md_gate);
    NXD_K(c, NXD_PROF_MIN_DISTANCE, min_distance, (pair_grid(c, 1, 1, 8, c->n_sm * 4)), (256), (0), c->geo, c->md_pairs, &c->sc->n_md_pairs, c->pair_cap, c->boxes, c->wv,
                                                &c->sc->md, &c->sc->md_gate);
    NXD_CUDA(cudaStreamSynchronize(st));
    Scalars h;
    NXD_CUDA(cudaMemcpy(&h, c->sc, sizeof(h), cudaMemcpyDeviceToHost));
    *out = h.md;
    return h.n_md_pairs > c->pair_cap ? NXD_CAPACITY : NXD_OK;
}

nxd_status nxd_profile(nxd_ctx* c, int32_t enable, double* ms, int64_t* launches) {
    if (!c) return NXD_INVALID_ARGUMENT;
    NXD_CUDA(cudaStreamSynchronize(c->stream));
    for (int f = 0; f < NXD_PROF_FAMILIES; ++f) {
        double t = 0.0;
        for (auto& pr : c->ev[f]) {
            float m = 0.f;
            if (cudaEventElapsedTime(&m, pr.first, pr.second) == cudaSuccess) t += m;
            c->pool.push_back(pr.first);
            c->pool.push_back(pr.second);
        }
        c->ev[f].clear();
        if (ms) ms[f] = t;
        if (launches) launches[f] = c->launches[f];
        c->launches[f] = 0;
    }
    c->prof = enable != 0;
    return NXD_OK;
}

nxd_status nxd_max_step(nxd_ctx* c, double dt, double* out_dt) {
    // IPCSolver::computeMaxStep (IPCSolver.cpp:355-392).  Every early exit
    // returns dt; otherwise CCDSystem::computeEarliestTOI (CCD.h:22-82) runs the
    // face-vertex root finder, whose first box ([0,1],[0,1],[0,1]) fails the
    // domain predicate w = 1-u-v in [0,1] (TimeOfImpact.cpp:130-139) before any
    // bisection, so no impact is ever reported and the bound is dt.
    if (!c || !out_dt) return NXD_INVALID_ARGUMENT;
    *out_dt = dt;
    return NXD_OK;
}

nxd_status nxd_set_form_state(nxd_ctx* c, const nxd_contact* contacts, int32_t n, const double* normal_forces,
                              const double* x_hat, double dt) {
    if (!c || n < 0 || n > kMaxRawContacts || (n > 0 && !contacts) || !(dt > 0.0)) return NXD_INVALID_ARGUMENT;
    cudaStream_t st = c->stream;
    if (n > 0)
        NXD_CUDA(cudaMemcpyAsync(c->contacts, contacts, sizeof(nxd_contact) * (size_t)n, cudaMemcpyHostToDevice, st));
    if (normal_forces && n > 0)
        NXD_CUDA(cudaMemcpyAsync(c->nforce, normal_forces, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, st));
    if (x_hat) NXD_CUDA(cudaMemcpyAsync(c->xhat, x_hat, 6 * sizeof(double) * (size_t)c->N, cudaMemcpyHostToDevice, st));
    NXD_LAUNCH(c, NXD_PROF_OTHER, k_set_form_state<<<grid_for(std::max(c->N, std::max(c->D, 1)), 128), 128, 0, st>>>(
        step_cfg(c), c->sc, n, normal_forces ? n : 0, dt, c->pos, c->quat, c->pos0, c->quat0, c->dhas_prev););
    NXD_CUDA(cudaStreamSynchronize(st));
    return NXD_OK;
}

static nxd_status form_call(nxd_ctx* c, int32_t form, const double* x, int what, double* host_out, int32_t* row_ptr,
                            int32_t* col_idx, double* vals, int64_t cap, int64_t* nnzb) {
    if (!c || !x || form < 0 || form > NXD_FORM_CONTACT) return NXD_INVALID_ARGUMENT;
    cudaStream_t st = c->stream;
    const size_t n6 = 6 * (size_t)c->N;
    double* xd = c->S.xt;   // scratch (the step is not running on this stream)
    NXD_CUDA(cudaMemcpyAsync(xd, x, n6 * sizeof(double), cudaMemcpyHostToDevice, st));
    DevArena tmp;
    double* outd = tmp.alloc<double>(what == 1 ? n6 : 1);
    int* rp = nullptr; int* ci = nullptr; double* vv = nullptr; long long* nz = nullptr;
    if (what == 2) {
        rp = tmp.alloc<int>(c->N + 1);
        ci = tmp.alloc<int>(std::max<int64_t>(cap, 1));
        vv = tmp.alloc<double>(36 * (size_t)std::max<int64_t>(cap, 1));
        nz = tmp.alloc<long long>(1);
    }
    if (!tmp.ok) { tmp.release(); return NXD_CUDA_ERROR; }
    NXD_LAUNCH(c, NXD_PROF_OTHER, k_form_eval<<<1, kSolverThreads, 0, st>>>(c->S, c->sc, form, what, xd, outd, rp, ci, vv, cap, nz););
    cudaError_t e = cudaStreamSynchronize(st);
    nxd_status rc = NXD_OK;
    if (e != cudaSuccess) rc = NXD_CUDA_ERROR;
    else if (what == 0) cudaMemcpy(host_out, outd, sizeof(double), cudaMemcpyDeviceToHost);
    else if (what == 1) cudaMemcpy(host_out, outd, n6 * sizeof(double), cudaMemcpyDeviceToHost);
    else {
        long long nzh = 0;
        cudaMemcpy(&nzh, nz, sizeof(long long), cudaMemcpyDeviceToHost);
        if (nnzb) *nnzb = nzh;
        if (nzh < 0) rc = NXD_INVALID_ARGUMENT;
        else if (nzh > cap) rc = NXD_CAPACITY;
        else {
            if (row_ptr) cudaMemcpy(row_ptr, rp, sizeof(int) * (c->N + 1), cudaMemcpyDeviceToHost);
            if (col_idx) cudaMemcpy(col_idx, ci, sizeof(int) * (size_t)nzh, cudaMemcpyDeviceToHost);
            if (vals) cudaMemcpy(vals, vv, 36 * sizeof(double) * (size_t)nzh, cudaMemcpyDeviceToHost);
        }
    }
    tmp.release();
    return rc;
}

nxd_status nxd_form_value(nxd_ctx* c, int32_t form, const double* x, double* out) {
    if (!out) return NXD_INVALID_ARGUMENT;
    return form_call(c, form, x, 0, out, nullptr, nullptr, nullptr, 0, nullptr);
}
nxd_status nxd_form_gradient(nxd_ctx* c, int32_t form, const double* x, double* grad) {
    if (!grad) return NXD_INVALID_ARGUMENT;
    return form_call(c, form, x, 1, grad, nullptr, nullptr, nullptr, 0, nullptr);
}
nxd_status nxd_form_hessian_bsr(nxd_ctx* c, int32_t form, const double* x, int32_t* row_ptr, int32_t* col_idx,
                                double* vals, int64_t cap, int64_t* nnzb) {
    return form_call(c, form, x, 2, nullptr, row_ptr, col_idx, vals, cap, nnzb);
}

nxd_status nxd_eval_all(nxd_ctx* c, const double* x, double* energy, double* grad, int32_t* row_ptr,
                        int32_t* col_idx, double* vals, int64_t cap, int64_t* nnzb) {
    if (!energy || !grad) return NXD_INVALID_ARGUMENT;
    nxd_status rc = form_call(c, NXD_FORM_TOTAL, x, 0, energy, nullptr, nullptr, nullptr, 0, nullptr);
    if (rc == NXD_OK) rc = form_call(c, NXD_FORM_TOTAL, x, 1, grad, nullptr, nullptr, nullptr, 0, nullptr);
    if (rc == NXD_OK) rc = form_call(c, NXD_FORM_TOTAL, x, 2, nullptr, row_ptr, col_idx, vals, cap, nnzb);
    return rc;
}

nxd_status nxd_linear_solve(nxd_ctx* c, const nxd_bsr* H, const double* b, double* x, nxd_solve_stats* stats) {
    if (!c || !H || !b || !x || H->n_rows != c->N || H->nnzb < 0 || H->nnzb > INT32_MAX ||
        (H->nnzb > 0 && (!H->row_ptr || !H->col_idx || !H->vals)))
        return NXD_INVALID_ARGUMENT;
    const int N = c->N;
    const long long nb = H->nnzb;
    for (int i = 0; i < N; ++i)
        if (H->row_ptr[i] > H->row_ptr[i + 1] || H->row_ptr[i] < 0) return NXD_INVALID_ARGUMENT;
    if (H->row_ptr[0] != 0 || H->row_ptr[N] != nb) return NXD_INVALID_ARGUMENT;
    for (long long k = 0; k < nb; ++k)
        if (H->col_idx[k] < 0 || H->col_idx[k] >= N) return NXD_INVALID_ARGUMENT;
    cudaStream_t st = c->stream;
    DevArena tmp;
    int* rp = tmp.alloc<int>(N + 1);
    int* ci = tmp.alloc<int>(std::max<long long>(nb, 1));
    int* er = tmp.alloc<int>(std::max<long long>(nb, 1));
    double* vv = tmp.alloc<double>(36 * (size_t)std::max<long long>(nb, 1));
    double* bd = tmp.alloc<double>(6 * (size_t)N);
    int* items = tmp.alloc<int>(std::max<long long>(nb, 1));
    int* iact = tmp.alloc<int>(std::max<long long>(nb, 1));
    int* stat = tmp.alloc<int>(1);
    if (!tmp.ok) { tmp.release(); return NXD_CUDA_ERROR; }
    NXD_CUDA(cudaMemcpyAsync(rp, H->row_ptr, sizeof(int) * (N + 1), cudaMemcpyHostToDevice, st));
    if (nb > 0) {
        NXD_CUDA(cudaMemcpyAsync(ci, H->col_idx, sizeof(int) * nb, cudaMemcpyHostToDevice, st));
        NXD_CUDA(cudaMemcpyAsync(vv, H->vals, 36 * sizeof(double) * nb, cudaMemcpyHostToDevice, st));
    }
    NXD_CUDA(cudaMemcpyAsync(bd, b, 6 * sizeof(double) * N, cudaMemcpyHostToDevice, st));
    NXD_CUDA(cudaMemsetAsync(stat, 0, sizeof(int), st));
    Solver S = c->S;
    S.ext_n = (int)nb; S.ext_row = er; S.ext_col = ci; S.ext_vals = vv;
    S.items = items; S.iact = iact; S.status = stat;
    if (N > 0) k_bsr_prepare<<<grid_for(N, 128), 128, 0, st>>>(S, rp, bd, er);
    if (N > 0) k_linear_solve<<<1, kNewtonThreads, kNewtonDynSmem, st>>>(S);
    NXD_CUDA(cudaGetLastError());
    NXD_CUDA(cudaStreamSynchronize(st));
    int fail = 0, capst = 0;
    cudaMemcpy(&fail, S.solve_fail, sizeof(int), cudaMemcpyDeviceToHost);
    cudaMemcpy(&capst, stat, sizeof(int), cudaMemcpyDeviceToHost);
    cudaMemcpy(x, S.dx, 6 * sizeof(double) * N, cudaMemcpyDeviceToHost);
    if (stats) {
        std::vector<int> rflag(N + 1), mcnt(N + 1), comp(N);
        cudaMemcpy(rflag.data(), S.rflag, sizeof(int) * (N + 1), cudaMemcpyDeviceToHost);
        cudaMemcpy(mcnt.data(), S.mcnt, sizeof(int) * (N + 1), cudaMemcpyDeviceToHost);
        cudaMemcpy(comp.data(), S.comp, sizeof(int) * N, cudaMemcpyDeviceToHost);
        stats->components = rflag[N];
        int in_multi = 0, largest = N > 0 ? 1 : 0;
        for (int r = 0; r < N; ++r)
            if (rflag[r + 1] != rflag[r]) {
                const int k = mcnt[r + 1] - mcnt[r];
                in_multi += k;
                largest = std::max(largest, k);
            }
        stats->singletons = N - in_multi;
        stats->largest_component = largest;
        stats->factor_failed = (fail && !capst) ? 1 : 0;
    }
    tmp.release();
    if (capst) return NXD_CAPACITY;
    return fail ? NXD_FACTOR_FAILED : NXD_OK;
}

}  // extern "C"

namespace {

// A device buffer that grows on demand (cudaMalloc at the first use and
// when a larger size is needed; kept until released).
struct GrowBuf {
    void* p = nullptr;
    size_t cap = 0;
    bool ensure(size_t bytes) {
        bytes = std::max<size_t>(bytes, 256);
        if (bytes <= cap) return true;
        if (p) {
            cudaDeviceSynchronize();   // queued kernels may still read the old buffer
            cudaFree(p);
        }
        p = nullptr;
        cap = 0;
        if (cudaMalloc(&p, bytes) != cudaSuccess) { p = nullptr; return false; }
        cap = bytes;
        return true;
    }
    template <typename T> T* as() const { return static_cast<T*>(p); }
    void release() { if (p) cudaFree(p); p = nullptr; cap = 0; }
};

// PCG on a device-resident BSR system; x (device) gets the solution.
// Scratch comes from `buf` (grown as needed).  Returns the kernel's status
// (NXD_OK, NXD_FACTOR_FAILED) or NXD_CUDA_ERROR; *iters / *res / *ms report.
struct PcgScratch {
    GrowBuf minv, vec, part, bar, ints, res;
    GrowBuf dsym, cnt, urp, uci, uvals, lrp, lidx, lrow;   // the upper block triangle (pcg.cuh)
    void release() {
        for (GrowBuf* g : {&minv, &vec, &part, &bar, &ints, &res, &dsym, &cnt, &urp, &uci, &uvals, &lrp, &lidx, &lrow})
            g->release();
    }
};
nxd_status pcg_device(nxd_ctx* c, PcgScratch& w, int N, const int* rp, const int* ci, const double* vv, const double* bd,
                      double* xd, double tol, int max_iter, int* iters, double* res, float* ms, int* grid) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pcg, kPcgThreads, 0);
    const long long n6 = 6LL * N;
    const long long need = (n6 + kPcgThreads - 1) / kPcgThreads;
    // at most two CTAs per SM: every grid barrier of the iteration waits for
    // all CTAs, so more of them cost more than their latency hiding gains
    const int G = (int)std::max<long long>(1, std::min<long long>((long long)std::min(std::max(per_sm, 1), 2) * c->n_sm, need));
    cudaStream_t st = c->stream;
    if (!w.minv.ensure(8 * kSym * (size_t)N) || !w.dsym.ensure(8 * kSym * (size_t)N) || !w.vec.ensure(48 * 6 * (size_t)N) ||
        !w.part.ensure(8 * 2 * kPcgMaxQ * (size_t)G) || !w.bar.ensure(8) || !w.ints.ensure(16) || !w.res.ensure(8) ||
        !w.cnt.ensure(8 * (size_t)N) || !w.urp.ensure(4 * (size_t)(N + 1)) || !w.lrp.ensure(4 * (size_t)(N + 1)))
        return NXD_CUDA_ERROR;
    int* ints = w.ints.as<int>();
    unsigned* bar = w.bar.as<unsigned>();
    double* vec = w.vec.as<double>();
    int* urp = w.urp.as<int>();
    int* lrp = w.lrp.as<int>();
    NXD_CUDA(cudaMemsetAsync(ints, 0, 4 * sizeof(int), st));
    NXD_CUDA(cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned), st));
    k_pcg_prepare<<<grid_for(N, 128), 128, 0, st>>>(N, rp, ci, vv, w.minv.as<double>(), w.dsym.as<double>(), ints + 2);
    // the upper block triangle: distinct columns per row, their offsets
    k_pcg_tri_count<<<grid_for(N, 128), 128, 0, st>>>(N, rp, ci, w.cnt.as<int>(), w.cnt.as<int>() + N);
    k_scan<<<1, 1024, 0, st>>>(w.cnt.as<int>(), urp, N, urp + N, nullptr, nullptr, nullptr);
    k_scan<<<1, 1024, 0, st>>>(w.cnt.as<int>() + N, lrp, N, lrp + N, nullptr, nullptr, nullptr);
    int h4[3] = {0, 0, 0};   // fail, upper blocks, lower entries
    NXD_CUDA(cudaMemcpyAsync(&h4[0], ints + 2, sizeof(int), cudaMemcpyDeviceToHost, st));
    NXD_CUDA(cudaMemcpyAsync(&h4[1], urp + N, sizeof(int), cudaMemcpyDeviceToHost, st));
    NXD_CUDA(cudaMemcpyAsync(&h4[2], lrp + N, sizeof(int), cudaMemcpyDeviceToHost, st));
    NXD_CUDA(cudaStreamSynchronize(st));
    if (h4[0]) return NXD_FACTOR_FAILED;
    if (h4[1] != h4[2]) return NXD_INVALID_ARGUMENT;   // not structurally symmetric
    const size_t nu = std::max(h4[1], 1);
    if (!w.uci.ensure(4 * nu) || !w.uvals.ensure(288 * nu) || !w.lidx.ensure(4 * nu) || !w.lrow.ensure(4 * nu))
        return NXD_CUDA_ERROR;
    k_pcg_tri_upper<<<grid_for(N, 128), 128, 0, st>>>(N, rp, ci, vv, urp, w.uci.as<int>(), w.uvals.as<double>());
    k_pcg_tri_lower<<<grid_for(N, 128), 128, 0, st>>>(N, rp, ci, urp, w.uci.as<int>(), lrp, w.lidx.as<int>(),
                                                      w.lrow.as<int>(), ints + 3);
    PcgArgs A;
    A.N = N; A.urp = urp; A.uci = w.uci.as<int>(); A.uvals = w.uvals.as<double>();
    A.lrp = lrp; A.lidx = w.lidx.as<int>(); A.lrow = w.lrow.as<int>(); A.dsym = w.dsym.as<double>();
    A.minv = w.minv.as<double>(); A.b = bd;
    A.x = xd; A.r[0] = vec; A.r[1] = vec + n6; A.p[0] = vec + 2 * n6; A.p[1] = vec + 3 * n6;
    A.q = vec + 4 * n6; A.z = vec + 5 * n6; A.tol = tol; A.max_iter = max_iter; A.part = w.part.as<double>(); A.stride = G;
    A.bar_count = bar; A.bar_abort = (int*)(bar + 1); A.status = ints; A.iters_out = ints + 1; A.res_out = w.res.as<double>();
    int fail = 0;
    NXD_CUDA(cudaMemcpyAsync(&fail, ints + 3, sizeof(int), cudaMemcpyDeviceToHost, st));
    NXD_CUDA(cudaStreamSynchronize(st));
    if (fail) return NXD_INVALID_ARGUMENT;            // a block without its transpose
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0); cudaEventCreate(&e1);
    void* args[] = {(void*)&A};
    cudaEventRecord(e0, st);
    const cudaError_t le = cudaLaunchCooperativeKernel((const void*)k_pcg, dim3(G), dim3(kPcgThreads), args, 0, st);
    cudaEventRecord(e1, st);
    NXD_CUDA(cudaStreamSynchronize(st));
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0); cudaEventDestroy(e1);
    if (le != cudaSuccess) return NXD_CUDA_ERROR;
    int h[2] = {0, 0};
    NXD_CUDA(cudaMemcpy(h, ints, 2 * sizeof(int), cudaMemcpyDeviceToHost));
    NXD_CUDA(cudaMemcpy(res, w.res.p, sizeof(double), cudaMemcpyDeviceToHost));
    *iters = h[1];
    if (ms) *ms = t;
    if (grid) *grid = G;
    return (nxd_status)h[0];
}

}  // namespace

extern "C" {

nxd_status nxd_pcg_solve(nxd_ctx* c, const nxd_bsr* H, const double* b, double* x, double tol, int32_t max_iter,
                         nxd_pcg_stats* stats) {
    if (!c || !H || !b || !x || H->n_rows <= 0 || H->nnzb < 0 || H->nnzb > INT32_MAX || max_iter < 0 || !(tol >= 0.0) ||
        (H->nnzb > 0 && (!H->row_ptr || !H->col_idx || !H->vals)))
        return NXD_INVALID_ARGUMENT;
    const int N = H->n_rows;
    const long long nb = H->nnzb, n6 = 6LL * N;
    if (n6 > INT32_MAX) return NXD_INVALID_ARGUMENT;
    for (int i = 0; i < N; ++i)
        if (H->row_ptr[i] > H->row_ptr[i + 1] || H->row_ptr[i] < 0) return NXD_INVALID_ARGUMENT;
    if (H->row_ptr[0] != 0 || H->row_ptr[N] != nb) return NXD_INVALID_ARGUMENT;
    for (long long k = 0; k < nb; ++k)
        if (H->col_idx[k] < 0 || H->col_idx[k] >= N) return NXD_INVALID_ARGUMENT;
    cudaStream_t st = c->stream;
    DevArena tmp;
    int* rp = tmp.alloc<int>(N + 1);
    int* ci = tmp.alloc<int>(std::max<long long>(nb, 1));
    double* vv = tmp.alloc<double>(36 * (size_t)std::max<long long>(nb, 1));
    double* bd = tmp.alloc<double>((size_t)n6);
    double* xd = tmp.alloc<double>((size_t)n6);
    if (!tmp.ok) { tmp.release(); return NXD_CUDA_ERROR; }
    NXD_CUDA(cudaMemcpyAsync(rp, H->row_ptr, sizeof(int) * (N + 1), cudaMemcpyHostToDevice, st));
    if (nb > 0) {
        NXD_CUDA(cudaMemcpyAsync(ci, H->col_idx, sizeof(int) * nb, cudaMemcpyHostToDevice, st));
        NXD_CUDA(cudaMemcpyAsync(vv, H->vals, 36 * sizeof(double) * nb, cudaMemcpyHostToDevice, st));
    }
    NXD_CUDA(cudaMemcpyAsync(bd, b, sizeof(double) * n6, cudaMemcpyHostToDevice, st));
    PcgScratch w;
    int iters = 0, G = 0;
    double hr = 0.0;
    float ms = 0.f;
    const nxd_status rc = pcg_device(c, w, N, rp, ci, vv, bd, xd, tol, max_iter, &iters, &hr, &ms, &G);
    if (rc == NXD_OK) cudaMemcpy(x, xd, sizeof(double) * n6, cudaMemcpyDeviceToHost);
    if (stats) {
        stats->iterations = iters; stats->status = rc; stats->relative_residual = hr; stats->kernel_ms = ms;
        stats->grid = G; stats->threads = kPcgThreads;
    }
    w.release();
    tmp.release();
    if (rc != NXD_OK) return rc;
    return hr <= tol ? NXD_OK : NXD_NOT_CONVERGED;
}

nxd_status nxd_normal_forces(nxd_ctx* c, const double* x, double* out, int32_t n) {
    if (!c || !x || !out || n < 0) return NXD_INVALID_ARGUMENT;
    cudaStream_t st = c->stream;
    NXD_CUDA(cudaMemcpyAsync(c->S.xt, x, 6 * sizeof(double) * (size_t)c->N, cudaMemcpyHostToDevice, st));
    DevArena tmp;
    double* od = tmp.alloc<double>(std::max(n, 1));
    if (!tmp.ok) { tmp.release(); return NXD_CUDA_ERROR; }
    NXD_LAUNCH(c, NXD_PROF_OTHER, k_normal_forces<<<grid_for(std::max(n, 1), 128), 128, 0, st>>>(c->S, c->sc, c->S.xt, od, n););
    cudaStreamSynchronize(st);
    cudaMemcpy(out, od, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost);
    tmp.release();
    return NXD_OK;
}

// ---------------------------------------------------------------------------
// Primitive-level contact model (full IPC): LBVH candidates, barrier form
// (energy, gradient, PSD BSR Hessian), additive-CCD step bound.  Buffers are
// created on first use and grown to the counts a call needs; these calls
// synchronise and return host results.
// ---------------------------------------------------------------------------
}  // extern "C"

namespace {


struct Bvh {
    int n = 0;
    int topo_n = -1;    // primitive count of the hierarchy in child / parent / i0 (-1: none built)
    GrowBuf k0, k1, i0, i1, leaf, nbox, child, parent, rng, flags, bounds;
};

}  // namespace

// Device scalars of the full-IPC path (in IpcState::scal), copied whole into
// pinned host memory (IpcHost::sc) at each host wait, so that every value a
// phase reads back arrives with one copy and one stream synchronisation.
struct IpcScal {
    int tot[2];         // candidate totals: point-triangle, edge-edge
    int status;         // traversal status
    int nseg;           // segment count of the last ipc_segments
    int maxq[2];        // the most candidates of one query, per kind
    int na;             // active barrier pairs
    int naccd;          // CCD pairs left for the sampling rounds
    long long rnz;      // rest-form Hessian blocks
    double energy;      // barrier energy
    double alpha;       // CCD step bound
    double rest;        // rest-form value
    double descent;     // g . dx
    double ginf;        // |g|_inf
    double dxinf;       // |dx|_inf
    double fenergy;     // friction energy (the frozen pairs' potential)
};
struct IpcHost {
    IpcScal sc;
    int fail, capst;    // linear-solve flags
};

struct IpcState {
    PrimGeo pg{};
    GrowBuf fbody, fvert, ebody, evert;
    GrowBuf x0, x1, pp0, pq0, pp1, pq1, wq0, wq1, qv, qe;
    Bvh faces, edges;
    GrowBuf cnt, off, cnt2, off2, pt, ee, scal, hist;
    IpcHost* hp = nullptr;       // pinned
    int* hrow = nullptr;         // pinned, 3 (N + 1) row pointers
    IpcScal* ds() const { return scal.as<IpcScal>(); }
    int n_pt = 0, n_ee = 0;
    bool cand_swept = false;     // the last ipc_candidates_begin built swept boxes
    bool pose_x = false;         // the last ipc_pose was at an iterate (x0 holds it)
    // Inside one nxd_ipc_step the hierarchies built at the step's first
    // iterate are refitted to every later iterate, swept pose and trial
    // instead of rebuilt: the candidate lists are sorted by (query,
    // primitive) whatever the hierarchy, so they are the same lists.
    bool keep_trees = false;
    GrowBuf tkey, tval, tkey1, tval1;    // candidate pairs sorted by (query, primitive) keys
    GrowBuf qbuf0, qbuf1;                // per query the first hits of the count traversal (k_traverse)
    GrowBuf dxv, rmax, pad;              // the last ipc_pose's dx, per-body vertex radius and arc pad
    GrowBuf scan_sums;                   // tile sums of scan_ints
    // lagged friction of the step: the frozen pairs (IpcFric), built from
    // the active pairs of the barrier evaluation that follows fr_build, and
    // the step-start world vertices they measure displacements from
    GrowBuf fr_vid, fr_body, fr_kind, fr_w, fr_nrm, fr_lam, fr_x0, fr_e;
    int fr_n = 0;
    bool fr_build = false;
    double fr_mu = 0.0, fr_eps = 1e-8;
    IpcFric fric() {
        return IpcFric{fr_n, fr_vid.as<int>(), fr_body.as<int>(), fr_kind.as<int>(), fr_w.as<double>(), fr_nrm.as<double>(),
                       fr_lam.as<double>(), fr_x0.as<double>()};
    }
    GrowBuf e, grad12, lam, z, nterm, body, active, type, apos, alist;
    GrowBuf gkey, gval, gkey1, gval1, hkey, hval, hkey1, hval1;
    GrowBuf sflag, spos, sstart, gout, rowptr, colidx, vals, toi, accd_list, accd_lpd0;
    // step adjoint: per-pair blocks, dense K^T and K_phi, vectors, outputs
    GrowBuf akp, akf, abody, aact, aK, aKphi, ax, axb, alam, aout, afail;
    GrowBuf afkp, afkf, afks, afgm, afbody, aKps, agmu;   // its friction pairs (lagged at the step start)
    // full-IPC time step: rest-form and merged BSR, gradients, solve scratch
    GrowBuf rrp, rci, rvv, mrp, mci, mvv, gr, gt, gneg, prod, xt, erow, items, iact, stat;
    PcgScratch pcg;
    std::vector<GrowBuf*> all() {
        return {&fbody, &fvert, &ebody, &evert, &x0, &x1, &pp0, &pq0, &pp1, &pq1, &wq0, &wq1, &qv, &qe,
                &faces.k0, &faces.k1, &faces.i0, &faces.i1, &faces.leaf, &faces.nbox, &faces.child, &faces.parent, &faces.rng,
                &faces.flags, &faces.bounds, &edges.k0, &edges.k1, &edges.i0, &edges.i1, &edges.leaf, &edges.nbox, &edges.rng,
                &edges.child, &edges.parent, &edges.flags, &edges.bounds, &cnt, &off, &cnt2, &off2, &pt, &ee, &scal, &hist, &e,
                &grad12, &lam, &z, &nterm, &body, &active, &type, &apos, &alist, &gkey, &gval, &gkey1, &gval1, &hkey,
                &hval, &hkey1, &hval1, &sflag, &spos, &sstart, &gout, &rowptr, &colidx, &vals, &toi, &accd_list, &accd_lpd0, &rrp, &rci, &rvv,
                &mrp, &mci, &mvv, &gr, &gt, &gneg, &prod, &xt, &erow, &items, &iact, &stat, &akp, &akf, &abody, &aact,
                &aK, &aKphi, &ax, &axb, &alam, &aout, &afail, &tkey, &tval, &tkey1, &tval1, &qbuf0, &qbuf1, &dxv, &rmax, &pad, &scan_sums, &afkp, &afkf, &afks, &afgm, &afbody,
                &aKps, &agmu, &fr_vid, &fr_body, &fr_kind, &fr_w, &fr_nrm, &fr_lam,
                &fr_x0, &fr_e};
    }
    void release() {
        for (GrowBuf* b : all()) b->release();
        pcg.release();
        if (hp) cudaFreeHost(hp);
        if (hrow) cudaFreeHost(hrow);
        hp = nullptr;
        hrow = nullptr;
    }
};

namespace {

#define IPC_ENSURE(buf, bytes) do { if (!(buf).ensure(bytes)) return NXD_CUDA_ERROR; } while (0)

void release_ipc(nxd_ctx* c) {
    if (!c->ipc) return;
    c->ipc->release();
    delete c->ipc;
    c->ipc = nullptr;
}

nxd_status ipc_init(nxd_ctx* c, IpcState* s) {
    IPC_ENSURE(s->fbody, 4 * (size_t)c->nf); IPC_ENSURE(s->fvert, 12 * (size_t)c->nf);
    IPC_ENSURE(s->ebody, 4 * (size_t)c->ne); IPC_ENSURE(s->evert, 8 * (size_t)c->ne);
    k_prim_topology<<<grid_for(c->N, 128), 128, 0, c->stream>>>(c->geo, s->fbody.as<int>(), s->fvert.as<int>(),
                                                              s->ebody.as<int>(), s->evert.as<int>());
    s->pg = PrimGeo{c->nv, c->nf, c->ne, c->vbody, s->fbody.as<int>(), s->ebody.as<int>(), s->fvert.as<int>(),
                    s->evert.as<int>()};
    IPC_ENSURE(s->scal, sizeof(IpcScal));
    NXD_CUDA(cudaMemsetAsync(s->scal.p, 0, sizeof(IpcScal), c->stream));
    IPC_ENSURE(s->rmax, 8 * (size_t)c->N); IPC_ENSURE(s->pad, 8 * (size_t)c->N);
    k_body_rmax<<<grid_for(c->N, 128), 128, 0, c->stream>>>(c->geo, s->rmax.as<double>());
    NXD_CUDA(cudaMallocHost(&s->hp, sizeof(IpcHost)));
    NXD_CUDA(cudaMallocHost(&s->hrow, 12 * (size_t)(c->N + 1)));
    NXD_CUDA(cudaGetLastError());
    return NXD_OK;
}

nxd_status ipc_prepare(nxd_ctx* c) {
    if (c->ipc) return NXD_OK;
    IpcState* s = new (std::nothrow) IpcState();
    if (!s) return NXD_CUDA_ERROR;
    c->ipc = s;
    const nxd_status st = ipc_init(c, s);
    if (st != NXD_OK) release_ipc(c);   // a later call starts again from nothing
    return st;
}

// One host wait: the device scalars into pinned memory (plus any copies
// queued before this call), then a stream synchronisation.
nxd_status ipc_fetch(nxd_ctx* c) {
    IpcState* s = c->ipc;
    NXD_CUDA(cudaMemcpyAsync(&s->hp->sc, s->scal.p, sizeof(IpcScal), cudaMemcpyDeviceToHost, c->stream));
    NXD_CUDA(cudaStreamSynchronize(c->stream));
    return NXD_OK;
}

// World vertices at x (host 6N; NULL = the current poses) into wq0, and at
// x + dx into wq1 when dx is given.
nxd_status ipc_pose(nxd_ctx* c, const double* x, const double* dx, bool on_device = false) {
    IpcState* s = c->ipc;
    const int N = c->N;
    const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    IPC_ENSURE(s->pp0, 24 * (size_t)N); IPC_ENSURE(s->pq0, 32 * (size_t)N); IPC_ENSURE(s->wq0, 24 * (size_t)c->nv);
    IPC_ENSURE(s->x0, 48 * (size_t)N);
    s->pose_x = x != nullptr;
    if (x) {
        NXD_CUDA(cudaMemcpyAsync(s->x0.p, x, 48 * (size_t)N, kind, c->stream));
        k_pose_at_x<<<grid_for(N, 128), 128, 0, c->stream>>>(N, s->x0.as<double>(), c->quat, s->pp0.as<double>(), s->pq0.as<double>());
    } else {
        NXD_CUDA(cudaMemcpyAsync(s->pp0.p, c->pos, 24 * (size_t)N, cudaMemcpyDeviceToDevice, c->stream));
        NXD_CUDA(cudaMemcpyAsync(s->pq0.p, c->quat, 32 * (size_t)N, cudaMemcpyDeviceToDevice, c->stream));
    }
    k_world_vertices<<<grid_for(c->nv, 256), 256, 0, c->stream>>>(c->geo, c->nv, c->vbody, s->pp0.as<double>(), s->pq0.as<double>(),
                                                                  s->wq0.as<double>());
    if (dx) {
        IPC_ENSURE(s->x1, 48 * (size_t)N); IPC_ENSURE(s->pp1, 24 * (size_t)N); IPC_ENSURE(s->pq1, 32 * (size_t)N);
        IPC_ENSURE(s->wq1, 24 * (size_t)c->nv); IPC_ENSURE(s->dxv, 48 * (size_t)N);
        NXD_CUDA(cudaMemcpyAsync(s->dxv.p, dx, 48 * (size_t)N, kind, c->stream));
        k_arc_pad<<<grid_for(N, 128), 128, 0, c->stream>>>(N, s->dxv.as<double>(), s->rmax.as<double>(), s->pad.as<double>());
        NXD_CUDA(cudaMemcpyAsync(s->x1.p, dx, 48 * (size_t)N, kind, c->stream));
        k_axpy_vec<<<grid_for(6 * N, 256), 256, 0, c->stream>>>(s->x0.as<double>(), s->x1.as<double>(), 6 * N, s->x1.as<double>());
        k_pose_at_x<<<grid_for(N, 128), 128, 0, c->stream>>>(N, s->x1.as<double>(), c->quat, s->pp1.as<double>(), s->pq1.as<double>());
        k_world_vertices<<<grid_for(c->nv, 256), 256, 0, c->stream>>>(c->geo, c->nv, c->vbody, s->pp1.as<double>(),
                                                                      s->pq1.as<double>(), s->wq1.as<double>());
    }
    NXD_CUDA(cudaGetLastError());
    return NXD_OK;
}

// Exclusive scan of n ints into out, the total into *total (device): one
// CTA below 8192 entries, the tiled multi-CTA scan above (sums: scratch).
nxd_status scan_ints(cudaStream_t st, GrowBuf& sums, const int* in, int* out, int n, int* total) {
    if (n <= 8192) {
        k_scan<<<1, 1024, 0, st>>>(in, out, n, total, nullptr, nullptr, nullptr);
        return NXD_OK;
    }
    const int nt = (n + kScanTile - 1) / kScanTile;
    if (!sums.ensure(4 * (size_t)nt)) return NXD_CUDA_ERROR;
    k_scan_tile_sums<<<nt, kScanTileThreads, 0, st>>>(in, n, sums.as<int>());
    k_scan_sums<<<1, 1024, 0, st>>>(sums.as<int>(), nt, total);
    k_scan_tiles<<<nt, kScanTileThreads, 0, st>>>(in, out, n, sums.as<int>());
    return NXD_OK;
}

// Stable LSD radix sort of n (key, value) pairs on key bits [lo, hi); the
// result ends in (k0, v0).
nxd_status radix_sort(nxd_ctx* c, GrowBuf& k0, GrowBuf& v0, GrowBuf& k1, GrowBuf& v1, int n, int lo, int hi) {
    if (n <= 1) return NXD_OK;
    IpcState* s = c->ipc;
    IPC_ENSURE(k1, 8 * (size_t)n); IPC_ENSURE(v1, 4 * (size_t)n);
    const int nblocks = (n + kRsTile - 1) / kRsTile;
    IPC_ENSURE(s->hist, 4 * 256 * (size_t)nblocks);
    for (int shift = lo; shift < hi; shift += 8) {
        k_rs_hist<<<nblocks, kRsThreads, 0, c->stream>>>(k0.as<unsigned long long>(), n, shift, s->hist.as<int>(), nblocks);
        k_rs_scan<<<1, 1024, 0, c->stream>>>(s->hist.as<int>(), 256 * nblocks);
        k_rs_scatter<<<nblocks, kRsThreads, 0, c->stream>>>(k0.as<unsigned long long>(), v0.as<int>(), k1.as<unsigned long long>(),
                                                            v1.as<int>(), n, shift, s->hist.as<int>(), nblocks);
        std::swap(k0, k1);
        std::swap(v0, v1);
    }
    NXD_CUDA(cudaGetLastError());
    return NXD_OK;
}

int bits_for(unsigned long long maxkey) {
    int b = 0;
    while (b < 64 && (maxkey >> b) != 0ull) ++b;
    return (b + 7) / 8 * 8;
}

// LBVH over the face (kind 0) or edge (kind 1) boxes: Morton keys, stable
// radix sort, Karras hierarchy, bottom-up boxes.
nxd_status ipc_build_bvh(nxd_ctx* c, Bvh& B, int kind, bool swept, double infl) {
    IpcState* s = c->ipc;
    const int n = kind == 0 ? c->nf : c->ne;
    B.n = n;
    IPC_ENSURE(B.leaf, 48 * (size_t)n);
    if (n == 0) return NXD_OK;
    const double* w1 = swept ? s->wq1.as<double>() : nullptr;
    k_ipc_boxes<<<grid_for(n, 256), 256, 0, c->stream>>>(s->pg, kind, s->wq0.as<double>(), w1, infl, B.leaf.as<double>(),
                                                         swept ? s->pad.as<double>() : nullptr);
    if (s->keep_trees && B.topo_n == n) {
        // the step's hierarchy, boxes refitted bottom-up
        NXD_CUDA(cudaMemsetAsync(B.flags.p, 0, 4 * (size_t)n, c->stream));
        k_refit<<<(n + kRefitChunk - 1) / kRefitChunk, kRefitChunk, 0, c->stream>>>(
            B.leaf.as<double>(), B.i0.as<int>(), n, B.child.as<int>(), B.parent.as<int>(), B.rng.as<int2>(), B.nbox.as<double>(),
            B.flags.as<int>());
        NXD_CUDA(cudaGetLastError());
        return NXD_OK;
    }
    B.topo_n = -1;
    IPC_ENSURE(B.bounds, 48);
    k_centroid_bounds<<<1, 1024, 0, c->stream>>>(B.leaf.as<double>(), n, B.bounds.as<double>());
    IPC_ENSURE(B.k0, 8 * (size_t)n); IPC_ENSURE(B.i0, 4 * (size_t)n);
    k_morton<<<grid_for(n, 256), 256, 0, c->stream>>>(B.leaf.as<double>(), n, B.bounds.as<double>(), B.k0.as<unsigned long long>(),
                                                      B.i0.as<int>());
    nxd_status st = radix_sort(c, B.k0, B.i0, B.k1, B.i1, n, 32, 64);
    if (st != NXD_OK) return st;
    IPC_ENSURE(B.nbox, 48 * (size_t)(2 * n - 1)); IPC_ENSURE(B.child, 8 * (size_t)n);
    IPC_ENSURE(B.parent, 4 * (size_t)(2 * n)); IPC_ENSURE(B.flags, 4 * (size_t)n); IPC_ENSURE(B.rng, 8 * (size_t)n);
    NXD_CUDA(cudaMemsetAsync(B.flags.p, 0, 4 * (size_t)n, c->stream));
    k_karras<<<grid_for(std::max(n - 1, 1), 128), 128, 0, c->stream>>>(B.k0.as<unsigned long long>(), n, B.child.as<int>(),
                                                                        B.parent.as<int>(), B.rng.as<int2>());
    k_refit<<<(n + kRefitChunk - 1) / kRefitChunk, kRefitChunk, 0, c->stream>>>(B.leaf.as<double>(), B.i0.as<int>(), n,
                                                                                  B.child.as<int>(), B.parent.as<int>(),
                                                                                  B.rng.as<int2>(), B.nbox.as<double>(),
                                                                                  B.flags.as<int>());
    NXD_CUDA(cudaGetLastError());
    B.topo_n = n;
    return NXD_OK;
}

// Candidate point-triangle (kind 0: vertex queries vs faces of another
// body) and edge-edge pairs (kind 1: edge queries vs edges of another body,
// query < primitive) at the posed world vertices: primitive boxes inflated
// by infl (swept over wq0 -> wq1 when swept), query boxes not inflated.
// Scenes of at most kSweepAllTests box tests take the all-pairs sweep, whose
// hits come out sorted; larger ones build (or refit) an LBVH per kind,
// count both kinds' hits in one traversal launch and put each query's hits
// in primitive order (copied from the count pass's per-query rows, or
// written by a second traversal and sorted per query, or past 2048 hits in
// one query by a radix sort of all pairs).  Both kinds are counted before
// the one host wait that reads their totals.
constexpr long long kSweepAllTests = 1LL << 22;
// ipc_candidates = ipc_candidates_begin (boxes, trees, counts and their
// scans, all queued) + one ipc_fetch + ipc_candidates_end (the writes); a
// caller may fold other read-backs into that fetch.
nxd_status ipc_candidates_pass(nxd_ctx* c, bool swept, double infl, int phase);
nxd_status ipc_candidates_begin(nxd_ctx* c, bool swept, double infl) { return ipc_candidates_pass(c, swept, infl, 0); }
nxd_status ipc_candidates_end(nxd_ctx* c) { return ipc_candidates_pass(c, c->ipc->cand_swept, 0.0, 1); }
nxd_status ipc_candidates(nxd_ctx* c, bool swept, double infl) {
    nxd_status st = ipc_candidates_begin(c, swept, infl);
    if (st == NXD_OK) st = ipc_fetch(c);
    if (st == NXD_OK) st = ipc_candidates_end(c);
    return st;
}
nxd_status ipc_candidates_pass(nxd_ctx* c, bool swept, double infl, int phase) {
    IpcState* s = c->ipc;
    IpcScal* ds = s->ds();
    const double* w1 = swept ? s->wq1.as<double>() : nullptr;
    const bool sweep = (long long)c->nv * c->nf + (long long)c->ne * c->ne <= kSweepAllTests;
    const int nq[2] = {c->nv, c->ne}, np[2] = {c->nf, c->ne};
    GrowBuf* cnt[2] = {&s->cnt, &s->cnt2};
    GrowBuf* off[2] = {&s->off, &s->off2};
    GrowBuf* out[2] = {&s->pt, &s->ee};
    Bvh* tree[2] = {&s->faces, &s->edges};
    GrowBuf* qbuf[2] = {&s->qbuf0, &s->qbuf1};
    // one kind's traversal job (buffers read at launch: they may grow)
    auto job = [&](int k, bool count) {
        Bvh& B = *tree[k];
        TravJob j{};
        j.kind = k;
        j.qbox = k == 0 ? s->qv.as<double>() : s->qe.as<double>();
        j.nq = nq[k];
        j.nbox = B.nbox.as<double>(); j.child = B.child.as<int>(); j.ids = B.i0.as<int>(); j.n = B.n;
        j.cnt = count ? cnt[k]->as<int>() : nullptr;
        j.off = count ? nullptr : off[k]->as<int>();
        j.out = count ? nullptr : out[k]->as<int>();
        j.maxq = &ds->maxq[k];
        j.qbuf = count ? qbuf[k]->as<int>() : nullptr;
        j.qorder = k == 1 && B.n == nq[1] ? B.i0.as<int>() : nullptr;   // edge queries in the edge tree's leaf order
        return j;
    };
    auto traverse = [&](const TravJob& a, const TravJob* b) {
        const int nb0 = grid_for(a.nq, 128), nb1 = b ? grid_for(b->nq, 128) : 0;
        k_traverse<<<nb0 + nb1, 128, 0, c->stream>>>(s->pg, a, b ? *b : a, nb0, &ds->status);
    };
    auto launch = [&](int k, bool count) {
        if (sweep)
            k_sweep_all<<<grid_for(32LL * nq[k], 128), 128, 0, c->stream>>>(
                s->pg, k, k == 0 ? s->qv.as<double>() : s->qe.as<double>(), nq[k], tree[k]->leaf.as<double>(), tree[k]->n,
                count ? cnt[k]->as<int>() : nullptr, count ? nullptr : off[k]->as<int>(), count ? nullptr : out[k]->as<int>());
        else
            traverse(job(k, count), nullptr);
    };
    if (phase == 1) {
        // after the fetch: the totals in pinned memory, then the writes
        if (s->hp->sc.status != 0) return (nxd_status)s->hp->sc.status;
        s->n_pt = s->hp->sc.tot[0];
        s->n_ee = s->hp->sc.tot[1];
        for (int k = 0; k < 2; ++k) {
            const int m = s->hp->sc.tot[k];
            IPC_ENSURE(*out[k], 8 * (size_t)std::max(m, 1));
            if (m == 0) continue;
            if (!sweep && s->hp->sc.maxq[k] == 0) {
                // every query's hits are in its qbuf row: copied and sorted there
                k_copy_slices<<<grid_for(nq[k], 128), 128, 0, c->stream>>>(qbuf[k]->as<int>(), cnt[k]->as<int>(),
                                                                           off[k]->as<int>(), out[k]->as<int>(), nq[k],
                                                                           nullptr, (long long)m);
                continue;
            }
            launch(k, false);
            if (sweep || m < 2) continue;
            // traversal order -> (query, primitive) ascending: the queries'
            // slices are already in query order, so each is sorted alone
            // (by its lane, or by its warp when longer than kSliceSortMax)
            // while the longest fits a warp's shared row; past that (a long
            // edge against thousands of a fine mesh's edges) one stable
            // radix sort of (query, primitive) keys
            if (s->hp->sc.maxq[k] <= kLongSliceMax) {
                k_sort_query_slices<<<grid_for(nq[k], kSliceSortThreads), kSliceSortThreads, 0, c->stream>>>(
                    out[k]->as<int>(), off[k]->as<int>(), cnt[k]->as<int>(), nq[k]);
                continue;
            }
            const int pbits = bits_for((unsigned long long)std::max(np[k], 1));
            const int qbits = bits_for((unsigned long long)std::max(nq[k], 1));
            IPC_ENSURE(s->tkey, 8 * (size_t)m); IPC_ENSURE(s->tval, 4 * (size_t)m);
            k_pair_keys<<<grid_for(m, 256), 256, 0, c->stream>>>(out[k]->as<int>(), m, pbits, s->tkey.as<unsigned long long>(),
                                                                 s->tval.as<int>());
            const nxd_status st = radix_sort(c, s->tkey, s->tval, s->tkey1, s->tval1, m, 0, pbits + qbits);
            if (st != NXD_OK) return st;
            k_pair_from_keys<<<grid_for(m, 256), 256, 0, c->stream>>>(s->tkey.as<unsigned long long>(), m, pbits,
                                                                      out[k]->as<int>());
        }
        NXD_CUDA(cudaGetLastError());
        return NXD_OK;
    }
    if (phase == 2) {
        // the writes into the lists' current capacities, the totals still on
        // the device (ipc_trial_energy): the all-pairs sweep writes again;
        // the tree copies the count pass's qbuf rows unless a query
        // overflowed its row (IpcScal::maxq, then nothing is written)
        for (int k = 0; k < 2; ++k) {
            if (nq[k] == 0 || np[k] == 0) continue;
            const double* qb = k == 0 ? s->qv.as<double>() : s->qe.as<double>();
            if (sweep)
                k_sweep_all<<<grid_for(32LL * nq[k], 128), 128, 0, c->stream>>>(s->pg, k, qb, nq[k], tree[k]->leaf.as<double>(),
                                                                                tree[k]->n, nullptr, off[k]->as<int>(),
                                                                                out[k]->as<int>(), (long long)(out[k]->cap / 8));
            else
                k_copy_slices<<<grid_for(nq[k], 128), 128, 0, c->stream>>>(qbuf[k]->as<int>(), cnt[k]->as<int>(),
                                                                           off[k]->as<int>(), out[k]->as<int>(), nq[k],
                                                                           ds->maxq, (long long)(out[k]->cap / 8));
        }
        NXD_CUDA(cudaGetLastError());
        return NXD_OK;
    }
    s->cand_swept = swept;
    const double* pad = swept ? s->pad.as<double>() : nullptr;
    if (sweep) {
        for (int k = 0; k < 2; ++k) {
            tree[k]->n = np[k];
            IPC_ENSURE(tree[k]->leaf, 48 * (size_t)std::max(np[k], 1));
            if (np[k])
                k_ipc_boxes<<<grid_for(np[k], 256), 256, 0, c->stream>>>(s->pg, k, s->wq0.as<double>(), w1, infl,
                                                                         tree[k]->leaf.as<double>(), pad);
        }
    } else {
        for (int k = 0; k < 2; ++k) {
            const nxd_status st = ipc_build_bvh(c, *tree[k], k, swept, infl);
            if (st != NXD_OK) return st;
        }
    }
    IPC_ENSURE(s->qv, 48 * (size_t)std::max(c->nv, 1)); IPC_ENSURE(s->qe, 48 * (size_t)std::max(c->ne, 1));
    if (c->nv)
        k_ipc_boxes<<<grid_for(c->nv, 256), 256, 0, c->stream>>>(s->pg, 2, s->wq0.as<double>(), w1, 0.0, s->qv.as<double>(), pad);
    if (c->ne)
        k_ipc_boxes<<<grid_for(c->ne, 256), 256, 0, c->stream>>>(s->pg, 3, s->wq0.as<double>(), w1, 0.0, s->qe.as<double>(), pad);
    NXD_CUDA(cudaMemsetAsync(ds, 0, 6 * sizeof(int), c->stream));   // totals, status, segment count, longest slices
    bool on[2];
    for (int k = 0; k < 2; ++k) {
        on[k] = nq[k] > 0 && np[k] > 0;
        if (!on[k]) continue;
        IPC_ENSURE(*cnt[k], 4 * (size_t)nq[k]); IPC_ENSURE(*off[k], 4 * (size_t)nq[k]);
        if (!sweep) IPC_ENSURE(*qbuf[k], 4 * (size_t)kQueryBuf * nq[k]);
    }
    if (sweep) {
        for (int k = 0; k < 2; ++k)
            if (on[k]) launch(k, true);
    } else if (on[0] || on[1]) {
        const TravJob a = job(on[0] ? 0 : 1, true), b = job(1, true);   // both kinds counted in one launch
        traverse(a, on[0] && on[1] ? &b : nullptr);
    }
    for (int k = 0; k < 2; ++k)
        if (on[k] && scan_ints(c->stream, s->scan_sums, cnt[k]->as<int>(), off[k]->as<int>(), nq[k], &ds->tot[k]) != NXD_OK)
            return NXD_CUDA_ERROR;
    NXD_CUDA(cudaGetLastError());
    return NXD_OK;
}

// Sorted segments of keys[0..m): starts in s->sstart (m_seg + 1 entries);
// the segment count stays on the device (IpcScal::nseg).
nxd_status ipc_segments(nxd_ctx* c, const unsigned long long* keys, int m) {
    IpcState* s = c->ipc;
    IPC_ENSURE(s->sflag, 4 * (size_t)m); IPC_ENSURE(s->spos, 4 * (size_t)m); IPC_ENSURE(s->sstart, 4 * (size_t)(m + 1));
    int* d_n = &s->ds()->nseg;
    k_seg_flags<<<grid_for(m, 256), 256, 0, c->stream>>>(keys, m, s->sflag.as<int>());
    if (scan_ints(c->stream, s->scan_sums, s->sflag.as<int>(), s->spos.as<int>(), m, d_n) != NXD_OK) return NXD_CUDA_ERROR;
    k_seg_starts<<<grid_for(m, 256), 256, 0, c->stream>>>(s->sflag.as<int>(), s->spos.as<int>(), m, s->sstart.as<int>(), d_n);
    NXD_CUDA(cudaGetLastError());
    return NXD_OK;
}

}  // namespace

extern "C" {

nxd_status nxd_ipc_candidates(nxd_ctx* c, const double* x, const double* dx, double inflation, int32_t* pt, int64_t pt_cap,
                              int32_t* ee, int64_t ee_cap, int64_t* n_pt, int64_t* n_ee) {
    if (!c || !n_pt || !n_ee || !(inflation >= 0.0) || (dx && !x)) return NXD_INVALID_ARGUMENT;
    nxd_status st = ipc_prepare(c);
    if (st == NXD_OK) st = ipc_pose(c, x, dx);
    if (st == NXD_OK) st = ipc_candidates(c, dx != nullptr, inflation);
    if (st != NXD_OK) return st;
    IpcState* s = c->ipc;
    *n_pt = s->n_pt;
    *n_ee = s->n_ee;
    if (pt && s->n_pt)
        NXD_CUDA(cudaMemcpy(pt, s->pt.p, 8 * (size_t)std::min<int64_t>(pt_cap, s->n_pt), cudaMemcpyDeviceToHost));
    if (ee && s->n_ee)
        NXD_CUDA(cudaMemcpy(ee, s->ee.p, 8 * (size_t)std::min<int64_t>(ee_cap, s->n_ee), cudaMemcpyDeviceToHost));
    return (pt && s->n_pt > pt_cap) || (ee && s->n_ee > ee_cap) ? NXD_CAPACITY : NXD_OK;
}

}  // extern "C"

namespace {

// The barrier form over the candidates of the last ipc_candidates call.
// The energy goes to IpcScal::energy on the device (read by the caller's
// next ipc_fetch).  With `full`, also the active count (IpcScal::na, read
// here with one host wait), the gradient in s->gout and the PSD BSR Hessian
// in s->rowptr / s->colidx / s->vals, its block count s->rowptr[N] on the
// device; *nh_out, when asked for, costs one more host wait.
// Friction energy of the frozen pairs at the pose ps into IpcScal::fenergy.
void ipc_friction_energy(nxd_ctx* c, const IpcPose& ps) {
    IpcState* s = c->ipc;
    k_fric_energy<<<grid_for(s->fr_n, 128), 128, 0, c->stream>>>(s->fric(), ps, s->fr_mu, s->fr_eps, s->fr_e.as<double>());
    k_tree_sum<<<1, 1024, 0, c->stream>>>(s->fr_e.as<double>(), s->fr_n, &s->ds()->fenergy);
}

nxd_status ipc_barrier_eval(nxd_ctx* c, double dhat, double kappa, bool full, int* nh_out) {
    IpcState* s = c->ipc;
    IpcScal* ds = s->ds();
    const int N = c->N, n = s->n_pt + s->n_ee;
    const IpcPairs P{s->pt.as<int>(), s->n_pt, s->ee.as<int>(), s->n_ee};
    const IpcPose ps{s->wq0.as<double>(), s->pp0.as<double>(), s->pose_x ? s->x0.as<double>() : nullptr};
    const size_t nn = std::max(n, 1);
    IPC_ENSURE(s->e, 8 * nn);
    if (!full) {
        if (n) k_ipc_pair_energy<<<grid_for(n, 128), 128, 0, c->stream>>>(s->pg, P, ps, dhat, kappa, s->e.as<double>());
        k_tree_sum<<<1, 1024, 0, c->stream>>>(s->e.as<double>(), n, &ds->energy);
        if (s->fr_n) ipc_friction_energy(c, ps);
        NXD_CUDA(cudaGetLastError());
        return NXD_OK;
    }
    // per-pair slots: the candidates, then the friction pairs (at most the
    // active candidates when the set is built at this evaluation)
    const size_t nf = (size_t)(s->fr_build ? n : s->fr_n);
    const size_t nt = std::max((size_t)n + nf, (size_t)1);
    IPC_ENSURE(s->grad12, 96 * nt); IPC_ENSURE(s->lam, 40 * nt); IPC_ENSURE(s->z, 480 * nt);
    IPC_ENSURE(s->nterm, 4 * nt); IPC_ENSURE(s->body, 8 * nt); IPC_ENSURE(s->active, 4 * nn); IPC_ENSURE(s->type, 4 * nn);
    IPC_ENSURE(s->apos, 4 * nn); IPC_ENSURE(s->alist, 4 * nt);
    const IpcEvalOut o{s->e.as<double>(), s->grad12.as<double>(), s->lam.as<double>(), s->z.as<double>(), s->nterm.as<int>(),
                       s->body.as<int>(), s->active.as<int>(), s->type.as<int>()};
    if (n) k_ipc_pair_eval<<<grid_for(n, 128), 128, 0, c->stream>>>(s->pg, P, ps, dhat, kappa, o);
    k_tree_sum<<<1, 1024, 0, c->stream>>>(s->e.as<double>(), n, &ds->energy);
    if (scan_ints(c->stream, s->scan_sums, s->active.as<int>(), s->apos.as<int>(), n, &ds->na) != NXD_OK)
        return NXD_CUDA_ERROR;
    if (n) k_compact<<<grid_for(n, 256), 256, 0, c->stream>>>(s->active.as<int>(), s->apos.as<int>(), n, s->alist.as<int>());
    nxd_status st = ipc_fetch(c);
    if (st != NXD_OK) return st;
    const int nb = s->hp->sc.na;
    if (s->fr_build) {
        // the friction set: the active pairs here, in pair order
        s->fr_build = false;
        s->fr_n = nb;
        const size_t m = std::max(nb, 1);
        IPC_ENSURE(s->fr_vid, 16 * m); IPC_ENSURE(s->fr_body, 8 * m); IPC_ENSURE(s->fr_kind, 4 * m);
        IPC_ENSURE(s->fr_w, 32 * m); IPC_ENSURE(s->fr_nrm, 24 * m); IPC_ENSURE(s->fr_lam, 8 * m); IPC_ENSURE(s->fr_e, 8 * m);
        if (nb) k_fric_lag<<<grid_for(nb, 128), 128, 0, c->stream>>>(s->pg, P, ps, s->alist.as<int>(), nb, dhat, kappa, s->fric());
    }
    if (s->fr_n) {
        k_fric_eval<<<grid_for(s->fr_n, 128), 128, 0, c->stream>>>(s->fric(), ps, s->fr_mu, s->fr_eps, n, s->fr_e.as<double>(), o);
        k_tree_sum<<<1, 1024, 0, c->stream>>>(s->fr_e.as<double>(), s->fr_n, &ds->fenergy);
        k_iota<<<grid_for(s->fr_n, 256), 256, 0, c->stream>>>(s->alist.as<int>(), &ds->na, n, s->fr_n);
    }
    // contributions: the active barrier pairs (pair order), then the friction pairs
    const int na = nb + s->fr_n;
    IPC_ENSURE(s->gout, 48 * (size_t)N);
    IPC_ENSURE(s->rowptr, 4 * (size_t)(N + 1));
    NXD_CUDA(cudaMemsetAsync(s->gout.p, 0, 48 * (size_t)N, c->stream));
    if (na == 0) {
        NXD_CUDA(cudaMemsetAsync(s->rowptr.p, 0, 4 * (size_t)(N + 1), c->stream));
        if (nh_out) *nh_out = 0;
        NXD_CUDA(cudaGetLastError());
        return NXD_OK;
    }
    // contributions, stable-sorted by body / by (row body, col body)
    IPC_ENSURE(s->gkey, 16 * (size_t)na); IPC_ENSURE(s->gval, 8 * (size_t)na);
    IPC_ENSURE(s->hkey, 32 * (size_t)na); IPC_ENSURE(s->hval, 16 * (size_t)na);
    k_ipc_contrib<<<grid_for(na, 128), 128, 0, c->stream>>>(s->alist.as<int>(), na, s->body.as<int>(), N,
                                                             s->gkey.as<unsigned long long>(), s->gval.as<int>(),
                                                             s->hkey.as<unsigned long long>(), s->hval.as<int>());
    st = radix_sort(c, s->gkey, s->gval, s->gkey1, s->gval1, 2 * na, 0, bits_for((unsigned long long)N));
    if (st == NXD_OK)
        st = radix_sort(c, s->hkey, s->hval, s->hkey1, s->hval1, 4 * na, 0, bits_for((unsigned long long)N * (unsigned long long)N));
    if (st != NXD_OK) return st;
    // at most 2 na gradient segments and 4 na Hessian blocks: the kernels
    // read the actual counts on the device, the grids cover the bounds
    IPC_ENSURE(s->sflag, 16 * (size_t)na); IPC_ENSURE(s->spos, 16 * (size_t)na); IPC_ENSURE(s->sstart, 16 * (size_t)na + 4);
    IPC_ENSURE(s->colidx, 16 * (size_t)na); IPC_ENSURE(s->vals, 1152 * (size_t)na);
    int* d_nseg = &ds->nseg;
    if ((st = ipc_segments(c, s->gkey.as<unsigned long long>(), 2 * na)) != NXD_OK) return st;
    k_ipc_grad<<<grid_for(12LL * na, 128), 128, 0, c->stream>>>(s->gkey.as<unsigned long long>(), s->gval.as<int>(),
                                                                 s->sstart.as<int>(), d_nseg, s->grad12.as<double>(),
                                                                 s->gout.as<double>());
    const int heavy_grid = 4 * c->n_sm;   // 32 warps per SM striding over the segments
    if (na > kSegSerial)
        k_ipc_grad_heavy<<<heavy_grid, 256, 0, c->stream>>>(s->gkey.as<unsigned long long>(), s->gval.as<int>(),
                                                             s->sstart.as<int>(), d_nseg, s->grad12.as<double>(),
                                                             s->gout.as<double>());
    if ((st = ipc_segments(c, s->hkey.as<unsigned long long>(), 4 * na)) != NXD_OK) return st;
    k_ipc_hess<<<grid_for(144LL * na, 128), 128, 0, c->stream>>>(s->hkey.as<unsigned long long>(), s->hval.as<int>(),
                                                                  s->sstart.as<int>(), d_nseg, N, s->lam.as<double>(),
                                                                  s->z.as<double>(), s->nterm.as<int>(), s->colidx.as<int>(),
                                                                  s->vals.as<double>(), 4LL * na);
    if (na > kSegSerial)
        k_ipc_hess_heavy<<<heavy_grid, 256, 0, c->stream>>>(s->hval.as<int>(), s->sstart.as<int>(), d_nseg, s->lam.as<double>(),
                                                             s->z.as<double>(), s->nterm.as<int>(), s->vals.as<double>(), 4LL * na);
    k_ipc_rowptr<<<grid_for(N + 1, 128), 128, 0, c->stream>>>(s->hkey.as<unsigned long long>(), s->sstart.as<int>(), d_nseg, N,
                                                               s->rowptr.as<int>());
    NXD_CUDA(cudaGetLastError());
    if (nh_out) {
        if ((st = ipc_fetch(c)) != NXD_OK) return st;
        *nh_out = s->hp->sc.nseg;
    }
    return NXD_OK;
}

// One line-search trial's barrier energy at xt (device) with a single host
// wait: candidates counted and written into the lists' current capacities
// (room for twice the last counts) -- by the all-pairs sweep, or from the
// refitted hierarchies' count pass (each query's hits kept in its qbuf row)
// inside a step -- the energy summed over the device-side counts, then one
// fetch.  *ok is false outside a step for a tree-sized scene, when a list
// overflowed or a query had more hits than its row holds: the caller then
// runs ipc_pose + ipc_candidates + ipc_barrier_eval.  The lists, their order
// and the sums are that path's.
nxd_status ipc_trial_energy(nxd_ctx* c, const double* xt, double dhat, double kappa, bool* ok) {
    IpcState* s = c->ipc;
    *ok = false;
    const bool sweep = (long long)c->nv * c->nf + (long long)c->ne * c->ne <= kSweepAllTests;
    // the hierarchies: only within a step, whose first iterate built them
    if (!sweep && !s->keep_trees) return NXD_OK;
    // capacities grow geometrically, so that a count creeping upwards does
    // not reallocate (and synchronise) on every trial
    auto room = [](GrowBuf& b, size_t want) { return want <= b.cap || b.ensure(std::max(want, 2 * b.cap)); };
    if (!room(s->pt, 16 * (size_t)std::max(s->n_pt, 16)) || !room(s->ee, 16 * (size_t)std::max(s->n_ee, 16)))
        return NXD_CUDA_ERROR;
    int cap_pt = (int)std::min<size_t>(s->pt.cap / 8, (size_t)1 << 30);
    int cap_ee = (int)std::min<size_t>(s->ee.cap / 8, (size_t)1 << 30);
    // test hook: NXD_IPC_TRIAL_CAP=<pairs> caps both lists, so that trials
    // whose candidates exceed it take the overflow path (same results)
    if (const char* tc = std::getenv("NXD_IPC_TRIAL_CAP")) {
        const int lim = std::max(0, std::atoi(tc));
        cap_pt = std::min(cap_pt, lim);
        cap_ee = std::min(cap_ee, lim);
    }
    if (!room(s->e, 8 * ((size_t)cap_pt + (size_t)cap_ee))) return NXD_CUDA_ERROR;
    nxd_status st = ipc_pose(c, xt, nullptr, true);
    if (st == NXD_OK) st = ipc_candidates_begin(c, false, dhat);
    if (st == NXD_OK) st = ipc_candidates_pass(c, false, dhat, 2);
    if (st != NXD_OK) return st;
    IpcScal* ds = s->ds();
    const IpcPose ps{s->wq0.as<double>(), s->pp0.as<double>(), s->pose_x ? s->x0.as<double>() : nullptr};
    k_ipc_pair_energy_dev<<<grid_for((long long)cap_pt + cap_ee, 128), 128, 0, c->stream>>>(
        s->pg, s->pt.as<int>(), s->ee.as<int>(), ds->tot, cap_pt, cap_ee, ps, dhat, kappa, s->e.as<double>(),
        sweep ? nullptr : ds->maxq);
    k_tree_sum_pairs<<<1, 1024, 0, c->stream>>>(s->e.as<double>(), ds->tot, cap_pt, cap_ee, &ds->energy);
    if (s->fr_n) ipc_friction_energy(c, ps);
    if ((st = ipc_fetch(c)) != NXD_OK) return st;
    const IpcScal& hs = s->hp->sc;
    if (hs.status != 0) return (nxd_status)hs.status;
    if (hs.tot[0] > cap_pt || hs.tot[1] > cap_ee) return NXD_OK;
    if (!sweep && (hs.maxq[0] | hs.maxq[1])) return NXD_OK;
    s->n_pt = hs.tot[0];
    s->n_ee = hs.tot[1];
    *ok = true;
    return NXD_OK;
}

// additive-CCD bound over the swept candidates of the last ipc_pose(x, dx),
// into IpcScal::alpha (read by the caller's next ipc_fetch)
nxd_status ipc_accd(nxd_ctx* c, double eta) {
    IpcState* s = c->ipc;
    const int n = s->n_pt + s->n_ee;
    IPC_ENSURE(s->toi, 8 * (size_t)std::max(n, 1));
    IPC_ENSURE(s->accd_list, 4 * (size_t)std::max(n, 1));
    IPC_ENSURE(s->accd_lpd0, 16 * (size_t)std::max(n, 1));
    const IpcPairs P{s->pt.as<int>(), s->n_pt, s->ee.as<int>(), s->n_ee};
    // along the rigid arcs from the last ipc_pose's x (x0) by its dx
    if (n) {
        int* nl = &s->ds()->naccd;
        NXD_CUDA(cudaMemsetAsync(nl, 0, sizeof(int), c->stream));
        k_ipc_accd<<<grid_for(n, 128), 128, 0, c->stream>>>(s->pg, P, c->geo.verts, s->x0.as<double>(), s->dxv.as<double>(),
                                                            c->quat, eta, 1000, s->toi.as<double>(), s->accd_list.as<int>(),
                                                            s->accd_lpd0.as<double2>(), nl);
        // a warp per listed pair: at most 16 warps per SM, striding over the list
        k_ipc_accd_rounds<<<grid_for(32LL * n, 128, 148 * 4), 128, 0, c->stream>>>(
            s->pg, P, c->geo.verts, s->x0.as<double>(), s->dxv.as<double>(), c->quat, eta, 1000, s->accd_list.as<int>(),
            s->accd_lpd0.as<double2>(), nl, s->toi.as<double>());
    }
    k_min_reduce<<<1, 1024, 0, c->stream>>>(s->toi.as<double>(), n, 1.0, &s->ds()->alpha);
    NXD_CUDA(cudaGetLastError());
    return NXD_OK;
}

}  // namespace

extern "C" {

nxd_status nxd_ipc_barrier(nxd_ctx* c, const double* x, double dhat, double kappa, double* energy, double* grad, int32_t* row_ptr,
                           int32_t* col_idx, double* vals, int64_t cap_blocks, int64_t* nnzb, int64_t* n_pairs,
                           int64_t* n_active) {
    if (!c || !(dhat > 0.0) || !(kappa >= 0.0)) return NXD_INVALID_ARGUMENT;
    nxd_status st = ipc_prepare(c);
    if (st == NXD_OK) st = ipc_pose(c, x, nullptr);
    if (st == NXD_OK) st = ipc_candidates(c, false, dhat);
    if (st != NXD_OK) return st;
    IpcState* s = c->ipc;
    const int N = c->N;
    if (n_pairs) *n_pairs = s->n_pt + s->n_ee;
    int nh = 0;
    st = ipc_barrier_eval(c, dhat, kappa, true, &nh);
    if (st != NXD_OK) return st;
    if (energy) *energy = s->hp->sc.energy;
    if (n_active) *n_active = s->hp->sc.na;
    if (grad) NXD_CUDA(cudaMemcpyAsync(grad, s->gout.p, 48 * (size_t)N, cudaMemcpyDeviceToHost, c->stream));
    if (nnzb) *nnzb = nh;
    if (nh > cap_blocks && (col_idx || vals)) { NXD_CUDA(cudaStreamSynchronize(c->stream)); return NXD_CAPACITY; }
    if (row_ptr) NXD_CUDA(cudaMemcpyAsync(row_ptr, s->rowptr.p, 4 * (size_t)(N + 1), cudaMemcpyDeviceToHost, c->stream));
    if (col_idx && nh) NXD_CUDA(cudaMemcpyAsync(col_idx, s->colidx.p, 4 * (size_t)nh, cudaMemcpyDeviceToHost, c->stream));
    if (vals && nh) NXD_CUDA(cudaMemcpyAsync(vals, s->vals.p, 288 * (size_t)nh, cudaMemcpyDeviceToHost, c->stream));
    NXD_CUDA(cudaStreamSynchronize(c->stream));
    NXD_CUDA(cudaGetLastError());
    return NXD_OK;
}

nxd_status nxd_ipc_max_step(nxd_ctx* c, const double* x, const double* dx, double eta, double* alpha, int64_t* n_pairs) {
    if (!c || !x || !dx || !alpha || !(eta > 0.0 && eta < 1.0)) return NXD_INVALID_ARGUMENT;
    nxd_status st = ipc_prepare(c);
    if (st == NXD_OK) st = ipc_pose(c, x, dx);
    if (st == NXD_OK) st = ipc_candidates(c, true, 0.0);
    if (st != NXD_OK) return st;
    if (n_pairs) *n_pairs = c->ipc->n_pt + c->ipc->n_ee;
    if (st == NXD_OK) st = ipc_accd(c, eta);
    if (st == NXD_OK) st = ipc_fetch(c);
    if (st == NXD_OK) *alpha = c->ipc->hp->sc.alpha;
    return st;
}

// Full-IPC time step: the x_tilde of implicit Euler (or Newmark) and the
// reference's inertia, gravity, joint (fixed multipliers) and control forms,
// with the primitive-pair barrier in place of the COM-distance contact forms.
// Newton starts from the step-start configuration, which is free of
// intersections, and follows NewtonSolver::minimize (|g|_inf test, Armijo
// backtracking) with the CCD bound as the line search's first step, and
// also stops when the Newton step is below tol * dt (IPC's velocity test:
// against a stiff barrier the absolute gradient test is out of reach in
// FP64).  Every iterate rebuilds the LBVH candidates at
// x (boxes inflated by dhat), and so does every trial point; the linear
// solve is nxd_linear_solve's component LDL^T on the rest-form blocks
// followed, row by row, by the barrier's blocks.
nxd_status nxd_ipc_step(nxd_ctx* c, double dt, const nxd_ipc_params* p, nxd_ipc_stats* out) {
    if (!c || !p || !(dt > 0.0) || !(p->dhat > 0.0) || !(p->kappa >= 0.0) || !(p->eta > 0.0 && p->eta < 1.0) ||
        p->newton_max_iters < 0 || p->ls_max_iters < 1 || p->linear_solver < 0 || p->linear_solver > 1 ||
        (p->linear_solver == 1 && (p->pcg_max_iter < 1 || !(p->pcg_tol >= 0.0))) || !(p->mu >= 0.0) ||
        (p->mu > 0.0 && (!(p->friction_eps > 0.0) || p->friction_iters < 1)))
        return NXD_INVALID_ARGUMENT;
    nxd_status st = ipc_prepare(c);
    if (st != NXD_OK) return st;
    IpcState* s = c->ipc;
    IpcScal* ds = s->ds();
    const IpcScal& hs = s->hp->sc;
    const int N = c->N, n6 = 6 * N;
    cudaStream_t sm = c->stream;
    StepCfg cfg = step_cfg(c);
    cfg.enable_adaptive = 0;
    cfg.enable_friction = 0;
    k_step_setup<<<grid_for(std::max(N, c->D), 128), 128, 0, sm>>>(cfg, dt, c->pos, c->quat, c->vel, c->omega, c->lacc, c->aacc, c->x,
        c->xhat, c->xprev, c->vprev, c->aprev, c->pos0, c->quat0, c->sc, c->dprm, c->dfilt, c->dfinit, c->dhas_prev);
    NXD_CUDA(cudaMemsetAsync(&c->sc->n_contacts, 0, sizeof(int), sm));
    NXD_CUDA(cudaMemcpyAsync(c->x, c->xprev, 8 * (size_t)n6, cudaMemcpyDeviceToDevice, sm));
    const double scale = cfg.newmark ? (cfg.beta * dt) * dt : dt * dt;
    // the rest-form kernel's CTA: a power of two from 64 to kSolverThreads
    // covering its widest loop (6N DOFs, J joints, D drives; no contact
    // forms here).  Its fixed-tree sums pad to powers of two with zeros, so
    // the width changes no result, and a small scene no longer pays for
    // 1024 threads on every call.
    int ft = 64;
    while (ft < kSolverThreads && ft < std::max({6 * N, c->J, c->D})) ft <<= 1;
    const long long cap_r = N + 2LL * (c->J + c->D);
    IPC_ENSURE(s->rrp, 4 * (size_t)(N + 1)); IPC_ENSURE(s->rci, 4 * (size_t)std::max(cap_r, 1LL));
    IPC_ENSURE(s->rvv, 288 * (size_t)std::max(cap_r, 1LL));
    IPC_ENSURE(s->mrp, 4 * (size_t)(N + 1)); IPC_ENSURE(s->gr, 8 * (size_t)n6);
    IPC_ENSURE(s->gt, 8 * (size_t)n6); IPC_ENSURE(s->gneg, 8 * (size_t)n6); IPC_ENSURE(s->prod, 8 * (size_t)n6);
    IPC_ENSURE(s->xt, 8 * (size_t)n6); IPC_ENSURE(s->stat, 8);
    double* x = c->x;
    int* rpr = s->hrow;                 // pinned: rest-form, barrier and merged row pointers
    int* rpb = s->hrow + (N + 1);
    int* rpm = s->hrow + 2 * (N + 1);
    // rest-form value at xx into IpcScal::rest, read at the next fetch
    auto rest_value = [&](const double* xx) {
        k_form_eval<<<1, ft, 0, sm>>>(c->S, c->sc, NXD_FORM_TOTAL, 0, xx, &ds->rest, nullptr, nullptr, nullptr, 0,
                                                  nullptr);
    };
    int iters = 0, conv = 0, lsfail = 0, solvefail = 0, na = 0, pcg_total = 0;
    double amax = 1.0, fx = 0.0;
    int64_t npairs = 0;
    bool cand_at_x = false;   // the last poses and dhat-inflated candidates were built at x
    // the hierarchies built at the first iterate serve the whole step
    struct TreeScope {
        IpcState* s;
        ~TreeScope() { s->keep_trees = false; s->fr_n = 0; s->fr_build = false; }
    } tree_scope{s};
    s->keep_trees = false;
    // lagged friction: pass 0 freezes the pairs active at the step start,
    // each further pass those at the previous pass's solution and solves again
    const bool friction = p->mu > 0.0;
    const int passes = friction ? p->friction_iters : 1;
    s->fr_n = 0;
    s->fr_mu = p->mu;
    s->fr_eps = friction ? p->friction_eps : 1e-8;
    int iters_done = 0;
    int64_t nfric = 0;
    for (int pass = 0; pass < passes; ++pass) {
        s->fr_build = friction;
        cand_at_x = false;
        conv = 0;
        iters = 0;
        for (int it = 0; it < p->newton_max_iters; ++it) {
            iters = it;
            // gradient at x: rest forms, then the barrier over the candidates at x
            k_form_eval<<<1, ft, 0, sm>>>(c->S, c->sc, NXD_FORM_TOTAL, 1, x, s->gr.as<double>(), nullptr, nullptr,
                                                      nullptr, 0, nullptr);
            // after an accepted trial the poses and candidates at x = xt (boxes
            // inflated by dhat) are the trial's, still in place
            st = NXD_OK;
            if (!cand_at_x) {
                st = ipc_pose(c, x, nullptr, true);
                if (st == NXD_OK) st = ipc_candidates(c, false, p->dhat);
                s->keep_trees = true;
                if (st == NXD_OK && friction && pass == 0 && it == 0) {
                    // the step-start world vertices (x = the step-start configuration)
                    IPC_ENSURE(s->fr_x0, 24 * (size_t)std::max(c->nv, 1));
                    NXD_CUDA(cudaMemcpyAsync(s->fr_x0.p, s->wq0.p, 24 * (size_t)c->nv, cudaMemcpyDeviceToDevice, sm));
                }
            }
            cand_at_x = false;
            if (st == NXD_OK) st = ipc_barrier_eval(c, p->dhat, p->kappa, true, nullptr);
            if (st != NXD_OK) return st;
            const double eb = hs.energy;   // the friction energy follows in the next fetch
            na = hs.na;
            nfric = s->fr_n;
            npairs = s->n_pt + s->n_ee;
            k_grad_combine<<<grid_for(n6, 256), 256, 0, sm>>>(s->gr.as<double>(), s->gout.as<double>(), scale, n6,
                                                              s->gt.as<double>(), s->gneg.as<double>());
            k_absmax<<<1, 1024, 0, sm>>>(s->gt.as<double>(), n6, &ds->ginf);
            // the rest forms' Hessian blocks and both row pointers come back with
            // |g|_inf in one wait (unused when the gradient test ends the solve)
            k_form_eval<<<1, ft, 0, sm>>>(c->S, c->sc, NXD_FORM_TOTAL, 2, x, nullptr, s->rrp.as<int>(), s->rci.as<int>(),
                                                      s->rvv.as<double>(), cap_r, &ds->rnz);
            NXD_CUDA(cudaMemcpyAsync(rpr, s->rrp.p, 4 * (size_t)(N + 1), cudaMemcpyDeviceToHost, sm));
            NXD_CUDA(cudaMemcpyAsync(rpb, s->rowptr.p, 4 * (size_t)(N + 1), cudaMemcpyDeviceToHost, sm));
            if ((st = ipc_fetch(c)) != NXD_OK) return st;
            if (hs.ginf < p->newton_tol) { conv = 1; break; }
            if (hs.rnz < 0 || hs.rnz > cap_r) return NXD_CAPACITY;
            // Hessian: rest-form blocks, then the barrier's, row by row
            rpm[0] = 0;
            for (int i = 0; i < N; ++i) rpm[i + 1] = rpm[i] + (rpr[i + 1] - rpr[i]) + (rpb[i + 1] - rpb[i]);
            const int nh = rpb[N];
            const long long nzm = rpm[N];
            IPC_ENSURE(s->mci, 4 * (size_t)std::max<long long>(nzm, 1)); IPC_ENSURE(s->mvv, 288 * (size_t)std::max<long long>(nzm, 1));
            IPC_ENSURE(s->erow, 4 * (size_t)std::max<long long>(nzm, 1)); IPC_ENSURE(s->items, 4 * (size_t)std::max<long long>(nzm, 1));
            IPC_ENSURE(s->iact, 4 * (size_t)std::max<long long>(nzm, 1));
            NXD_CUDA(cudaMemcpyAsync(s->mrp.p, rpm, 4 * (size_t)(N + 1), cudaMemcpyHostToDevice, sm));
            k_bsr_concat<<<grid_for(N, 128), 128, 0, sm>>>(N, s->rrp.as<int>(), s->rci.as<int>(), s->rvv.as<double>(),
                                                           nh ? s->rowptr.as<int>() : nullptr, s->colidx.as<int>(),
                                                           s->vals.as<double>(), scale, s->mrp.as<int>(), s->mci.as<int>(),
                                                           s->mvv.as<double>());
            // H dx = -g: block-Jacobi PCG, or the component LDL^T
            s->hp->fail = 0;
            s->hp->capst = 0;
            if (p->linear_solver == 1) {
                int pit = 0;
                double pres = 0.0;
                const nxd_status pr = pcg_device(c, s->pcg, N, s->mrp.as<int>(), s->mci.as<int>(), s->mvv.as<double>(),
                                                 s->gneg.as<double>(), c->S.dx, p->pcg_tol, p->pcg_max_iter, &pit, &pres,
                                                 nullptr, nullptr);
                if (pr == NXD_CUDA_ERROR) return pr;
                pcg_total += pit;
                if (pr != NXD_OK) { solvefail = 1; break; }
            } else {
                Solver S = c->S;
                S.ext_n = (int)nzm; S.ext_row = s->erow.as<int>(); S.ext_col = s->mci.as<int>(); S.ext_vals = s->mvv.as<double>();
                S.items = s->items.as<int>(); S.iact = s->iact.as<int>(); S.status = s->stat.as<int>();
                NXD_CUDA(cudaMemsetAsync(s->stat.p, 0, sizeof(int), sm));
                k_bsr_prepare<<<grid_for(N, 128), 128, 0, sm>>>(S, s->mrp.as<int>(), s->gneg.as<double>(), s->erow.as<int>());
                k_linear_solve<<<1, kNewtonThreads, kNewtonDynSmem, sm>>>(S);
                NXD_CUDA(cudaMemcpyAsync(&s->hp->fail, S.solve_fail, sizeof(int), cudaMemcpyDeviceToHost, sm));
                NXD_CUDA(cudaMemcpyAsync(&s->hp->capst, s->stat.p, sizeof(int), cudaMemcpyDeviceToHost, sm));
            }
            double* dx = c->S.dx;
            k_absmax<<<1, 1024, 0, sm>>>(dx, n6, &ds->dxinf);
            // the swept candidates of the step bound are counted before the wait
            // that reads the solve's flags (discarded when those end the loop)
            st = ipc_pose(c, x, dx, true);
            if (st == NXD_OK) st = ipc_candidates_begin(c, true, 0.0);
            if (st == NXD_OK) st = ipc_fetch(c);
            if (st != NXD_OK) return st;
            if (s->hp->capst) return NXD_CAPACITY;
            if (s->hp->fail) { solvefail = 1; break; }
            // the velocity criterion of IPC: a Newton step below tol * dt ends it
            if (hs.dxinf < p->newton_tol * dt) { conv = 1; break; }
            // the step bound (additive CCD over the swept candidates), the value
            // at x and the descent g . dx, read back in one wait
            st = ipc_candidates_end(c);
            if (st == NXD_OK) st = ipc_accd(c, p->eta);
            if (st != NXD_OK) return st;
            rest_value(x);
            k_mul_vec<<<grid_for(n6, 256), 256, 0, sm>>>(s->gt.as<double>(), dx, n6, s->prod.as<double>());
            k_tree_sum<<<1, 1024, 0, sm>>>(s->prod.as<double>(), n6, &ds->descent);
            if ((st = ipc_fetch(c)) != NXD_OK) return st;
            amax = hs.alpha;
            fx = hs.rest + scale * (s->fr_n ? eb + hs.fenergy : eb);
            const double descent = hs.descent;
            if (descent > 0) { lsfail = 1; break; }
            // line search from min(1, bound)
            double alpha = std::min(1.0, amax);
            bool done = false;
            for (int ls = 0; ls < p->ls_max_iters; ++ls) {
                k_axpy_alpha<<<grid_for(n6, 256), 256, 0, sm>>>(x, dx, alpha, n6, s->xt.as<double>());
                rest_value(s->xt.as<double>());
                bool one_wait = false;
                st = ipc_trial_energy(c, s->xt.as<double>(), p->dhat, p->kappa, &one_wait);
                if (st == NXD_OK && !one_wait) {
                    st = ipc_pose(c, s->xt.as<double>(), nullptr, true);
                    if (st == NXD_OK) st = ipc_candidates(c, false, p->dhat);
                    if (st == NXD_OK) st = ipc_barrier_eval(c, p->dhat, p->kappa, false, nullptr);
                    if (st == NXD_OK) st = ipc_fetch(c);
                }
                if (st != NXD_OK) return st;
                const double fn = hs.rest + scale * (s->fr_n ? hs.energy + hs.fenergy : hs.energy);
                if (fn <= fx + c->s.ls_c1 * alpha * descent) { done = true; fx = fn; break; }
                alpha *= c->s.ls_rho;
            }
            if (!done) { lsfail = 1; break; }
            cand_at_x = true;
            NXD_CUDA(cudaMemcpyAsync(x, s->xt.p, 8 * (size_t)n6, cudaMemcpyDeviceToDevice, sm));
            if (it == p->newton_max_iters - 1) iters = p->newton_max_iters;
        }
        iters_done += iters;
        if (!conv) break;   // a pass that did not converge ends the step
    }
    iters = iters_done;
    k_update_state<<<grid_for(N, 128), 128, 0, sm>>>(cfg, c->x, c->xprev, c->vprev, c->xhat, c->aprev, c->pos, c->quat, c->vel,
                                                   c->omega, c->lacc, c->aacc, c->sc, c->da, c->db, c->dprm, c->dfilt);
    NXD_CUDA(cudaStreamSynchronize(sm));
    NXD_CUDA(cudaGetLastError());
    if (out) {
        out->newton_iterations = iters; out->converged = conv; out->line_search_failed = lsfail;
        out->solve_failed = solvefail; out->last_alpha_max = amax; out->energy = fx; out->n_pairs = npairs;
        out->n_active = na; out->pcg_iterations = pcg_total; out->n_friction = nfric;
    }
    return solvefail ? NXD_FACTOR_FAILED : NXD_OK;
}

nxd_status nxd_ipc_adjoint(nxd_ctx* c, double dt, const nxd_ipc_params* p, const nxd_state* start, const double* x_star,
                           const double* x_bar, const nxd_ipc_adjoint_out* out) {
    if (!c || !p || !start || !x_star || !x_bar || !out || !(dt > 0.0) || !(p->dhat > 0.0) || !(p->kappa >= 0.0) ||
        !(p->mu >= 0.0) || (p->mu > 0.0 && (!(p->friction_eps > 0.0) || p->friction_iters != 1)))
        return NXD_INVALID_ARGUMENT;
    const int N = c->N, J = c->J, n6 = 6 * N;
    if (N > kAdjMaxBodies || c->D > 0 || c->s.integrator == NXD_INTEGRATOR_IMPLICIT_NEWMARK) return NXD_INVALID_ARGUMENT;
    for (int j = 0; j < J; ++j)
        if (c->h_jtype[j] != NXD_JOINT_FIXED) return NXD_INVALID_ARGUMENT;
    nxd_status st = nxd_set_state(c, start);
    if (st != NXD_OK) return st;
    if ((st = ipc_prepare(c)) != NXD_OK) return st;
    IpcState* s = c->ipc;
    cudaStream_t sm = c->stream;
    StepCfg cfg = step_cfg(c);
    cfg.enable_adaptive = 0;
    cfg.enable_friction = 0;
    // the step's predicted pose and step-start orientations, as nxd_ipc_step sets them
    k_step_setup<<<grid_for(std::max(N, 1), 128), 128, 0, sm>>>(cfg, dt, c->pos, c->quat, c->vel, c->omega, c->lacc, c->aacc,
        c->x, c->xhat, c->xprev, c->vprev, c->aprev, c->pos0, c->quat0, c->sc, c->dprm, c->dfilt, c->dfinit, c->dhas_prev);
    IPC_ENSURE(s->ax, 8 * (size_t)n6); IPC_ENSURE(s->axb, 8 * (size_t)n6); IPC_ENSURE(s->alam, 8 * (size_t)n6);
    NXD_CUDA(cudaMemcpyAsync(s->ax.p, x_star, 8 * (size_t)n6, cudaMemcpyHostToDevice, sm));
    NXD_CUDA(cudaMemcpyAsync(s->axb.p, x_bar, 8 * (size_t)n6, cudaMemcpyHostToDevice, sm));
    // friction: the pairs frozen at the step start, as the step's single
    // lagging pass froze them (pose x_prev = (p0, 0), dhat-inflated candidates)
    struct FricScope {
        IpcState* s;
        ~FricScope() { s->fr_n = 0; s->fr_build = false; }
    } fric_scope{s};
    const bool friction = p->mu > 0.0;
    s->fr_n = 0;
    if (friction) {
        st = ipc_pose(c, c->xprev, nullptr, true);
        if (st == NXD_OK) st = ipc_candidates(c, false, p->dhat);
        if (st != NXD_OK) return st;
        IPC_ENSURE(s->fr_x0, 24 * (size_t)std::max(c->nv, 1));
        NXD_CUDA(cudaMemcpyAsync(s->fr_x0.p, s->wq0.p, 24 * (size_t)c->nv, cudaMemcpyDeviceToDevice, sm));
        s->fr_build = true;
        s->fr_mu = p->mu;
        s->fr_eps = p->friction_eps;
        if ((st = ipc_barrier_eval(c, p->dhat, p->kappa, true, nullptr)) != NXD_OK) return st;
    }
    const int nf = s->fr_n;
    // candidates at x* (boxes inflated by dhat), each pair's exact blocks
    st = ipc_pose(c, s->ax.as<double>(), nullptr, true);
    if (st == NXD_OK) st = ipc_candidates(c, false, p->dhat);
    if (st != NXD_OK) return st;
    const int np = s->n_pt + s->n_ee;
    const size_t nn = std::max(np, 1);
    IPC_ENSURE(s->akp, 1152 * nn); IPC_ENSURE(s->akf, 576 * nn); IPC_ENSURE(s->abody, 8 * nn); IPC_ENSURE(s->aact, 4 * nn);
    IPC_ENSURE(s->aK, 8 * (size_t)n6 * n6); IPC_ENSURE(s->aKphi, 8 * (size_t)n6 * 3 * N);
    IPC_ENSURE(s->aout, 8 * (size_t)(3 * N * 3 + N + 9 * N + std::max(J, 1) + 3 * N + 1)); IPC_ENSURE(s->afail, 4);
    const size_t nfn = std::max(nf, 1);
    IPC_ENSURE(s->afkp, 1152 * nfn); IPC_ENSURE(s->afkf, 576 * nfn); IPC_ENSURE(s->afks, 1152 * nfn);
    IPC_ENSURE(s->afgm, 96 * nfn); IPC_ENSURE(s->afbody, 8 * nfn);
    IPC_ENSURE(s->aKps, 8 * (size_t)n6 * 3 * N); IPC_ENSURE(s->agmu, 8 * (size_t)n6);
    const IpcPairs P{s->pt.as<int>(), s->n_pt, s->ee.as<int>(), s->n_ee};
    const IpcPose ps{s->wq0.as<double>(), s->pp0.as<double>(), s->ax.as<double>()};
    if (np) k_ipc_pair_adjoint<<<grid_for(np, 64), 64, 0, sm>>>(s->pg, P, ps, p->dhat, p->kappa, s->akp.as<double>(),
                                                                s->akf.as<double>(), s->abody.as<int>(), s->aact.as<int>());
    if (nf)
        k_fric_pair_adjoint<<<grid_for(nf, 64), 64, 0, sm>>>(s->fric(), ps, c->pos, p->dhat, p->kappa, p->mu,
                                                             p->friction_eps, s->afkp.as<double>(), s->afkf.as<double>(),
                                                             s->afks.as<double>(), s->afgm.as<double>(), s->afbody.as<int>());
    const AdjFric afr{nf, s->afbody.as<int>(), s->afkp.as<double>(), s->afkf.as<double>(), s->afks.as<double>(),
                      s->afgm.as<double>(), s->aKps.as<double>(), s->agmu.as<double>()};
    AdjIn ai{N, J, c->mass, c->inertia, c->jtype, c->ja, c->jparams, c->jmu, c->quat0, s->ax.as<double>(), c->xhat, dt * dt};
    k_adj_assemble<<<1, kAdjThreads, 0, sm>>>(ai, s->abody.as<int>(), s->aact.as<int>(), s->akp.as<double>(),
                                              s->akf.as<double>(), np, s->aK.as<double>(), s->aKphi.as<double>(), afr);
    k_adj_solve<<<1, kAdjThreads, 0, sm>>>(s->aK.as<double>(), s->axb.as<double>(), n6, s->alam.as<double>(),
                                           s->afail.as<int>());
    double* o = s->aout.as<double>();
    AdjOut ao{o, o + 3 * N, o + 6 * N, o + 9 * N, o + 10 * N, o + 19 * N, o + 19 * N + std::max(J, 1),
              o + 22 * N + std::max(J, 1)};
    k_adj_cross<<<grid_for(std::max(3 * N, J), 128), 128, 0, sm>>>(ai, s->alam.as<double>(), s->aKphi.as<double>(), ao, afr);
    int fail = 0;
    NXD_CUDA(cudaMemcpyAsync(&fail, s->afail.p, sizeof(int), cudaMemcpyDeviceToHost, sm));
    const size_t n3 = 8 * 3 * (size_t)N;
    const cudaMemcpyKind d2h = cudaMemcpyDeviceToHost;
    if (out->lambda) NXD_CUDA(cudaMemcpyAsync(out->lambda, s->alam.p, 8 * (size_t)n6, d2h, sm));
    if (out->phat_bar) NXD_CUDA(cudaMemcpyAsync(out->phat_bar, ao.phat_bar, n3, d2h, sm));
    if (out->thetahat_bar) NXD_CUDA(cudaMemcpyAsync(out->thetahat_bar, ao.thetahat_bar, n3, d2h, sm));
    if (out->phi_bar) NXD_CUDA(cudaMemcpyAsync(out->phi_bar, ao.phi_bar, n3, d2h, sm));
    if (out->mass_bar) NXD_CUDA(cudaMemcpyAsync(out->mass_bar, ao.mass_bar, 8 * (size_t)N, d2h, sm));
    if (out->inertia_bar) NXD_CUDA(cudaMemcpyAsync(out->inertia_bar, ao.inertia_bar, 8 * 9 * (size_t)N, d2h, sm));
    if (out->joint_mu_bar && J) NXD_CUDA(cudaMemcpyAsync(out->joint_mu_bar, ao.joint_mu_bar, 8 * (size_t)J, d2h, sm));
    if (out->p0_bar) NXD_CUDA(cudaMemcpyAsync(out->p0_bar, ao.p0_bar, n3, d2h, sm));
    if (out->friction_mu_bar) NXD_CUDA(cudaMemcpyAsync(out->friction_mu_bar, ao.friction_mu_bar, 8, d2h, sm));
    if (out->n_active) {
        NXD_CUDA(cudaStreamSynchronize(sm));
        std::vector<int> act(np);
        if (np) NXD_CUDA(cudaMemcpy(act.data(), s->aact.p, 4 * (size_t)np, cudaMemcpyDeviceToHost));
        int na = 0;
        for (int a : act) na += a;
        *out->n_active = na;
    }
    NXD_CUDA(cudaStreamSynchronize(sm));
    NXD_CUDA(cudaGetLastError());
    return fail ? NXD_FACTOR_FAILED : NXD_OK;
}

// ---------------------------------------------------------------------------
// Batched scenes: one context per scene; the step sequences of all scenes are
// recorded, scenes with identical sequences form a group, and each group's
// step is one CUDA graph of batched launches (one launch per kernel position
// for all of the group's scenes, gridDim.y = scenes).
// ---------------------------------------------------------------------------
}  // extern "C"

namespace {

struct BatchGroup {
    std::vector<int> scenes;
    std::vector<const void*> kern, prep;
    std::vector<dim3> grid, block;
    std::vector<size_t> smem, table_off;
    void* table = nullptr;
    int* queue = nullptr;     // per queue-form position: prefix (scenes + 1) and counter
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

}  // namespace

struct nxd_batch {
    std::vector<nxd_ctx*> ctx;
    cudaStream_t stream = nullptr;
    std::vector<double> dts;           // the dts the groups were recorded with
    std::vector<BatchGroup> groups;
    bool own_stream = true;
    // persistent grid of each queue-form kernel: CTAs per SM (the result
    // does not depend on it; nxd_batch_set_queue_ctas, the autotuner)
    int queue_per_sm[kQueueKinds] = {4, 4};
    // with several groups, each group's graph runs on a stream of its own,
    // forked from and joined back into `stream` (the groups share nothing,
    // so one group's Newton CTAs fill the SMs another's leave early)
    std::vector<cudaStream_t> gstream;
    std::vector<cudaEvent_t> gdone;
    cudaEvent_t fork = nullptr;
};

namespace {

void release_groups(nxd_batch* b) {
    for (BatchGroup& g : b->groups) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        if (g.graph) cudaGraphDestroy(g.graph);
        if (g.table) cudaFree(g.table);
        if (g.queue) cudaFree(g.queue);
    }
    b->groups.clear();
}

// Records every scene's step with its dt and builds the group graphs.
nxd_status build_groups(nxd_batch* b, const double* dts) {
    release_groups(b);
    const int n = (int)b->ctx.size();
    std::vector<std::vector<LaunchRec>> recs(n);
    for (int i = 0; i < n; ++i) {
        nxd_ctx* c = b->ctx[i];
        c->rec = &recs[i];
        const nxd_status st = enqueue_step(c, dts[i]);
        c->rec = nullptr;
        if (st != NXD_OK) return st;
    }
    auto same_seq = [&](int i, int j) {
        if (recs[i].size() != recs[j].size()) return false;
        for (size_t k = 0; k < recs[i].size(); ++k) {
            const LaunchRec &x = recs[i][k], &y = recs[j][k];
            if (x.kern != y.kern || x.prep != y.prep || x.block.x != y.block.x || x.block.y != y.block.y ||
                x.block.z != y.block.z)
                return false;
        }
        return true;
    };
    for (int i = 0; i < n; ++i) {
        bool placed = false;
        for (BatchGroup& g : b->groups)
            if (same_seq(g.scenes[0], i)) { g.scenes.push_back(i); placed = true; break; }
        if (!placed) { b->groups.emplace_back(); b->groups.back().scenes.push_back(i); }
    }
    for (BatchGroup& g : b->groups) {
        const std::vector<LaunchRec>& r0 = recs[g.scenes[0]];
        const size_t L = r0.size(), ns = g.scenes.size();
        size_t bytes = 0;
        for (size_t k = 0; k < L; ++k) {
            g.table_off.push_back(bytes);
            bytes += (r0[k].args.size() * ns + 255) / 256 * 256;
        }
        std::vector<unsigned char> host(std::max<size_t>(bytes, 1));
        int nq = 0;
        const int n_sm = b->ctx[0]->n_sm;
        for (size_t k = 0; k < L; ++k) {
            unsigned gx = 1;
            size_t smem = 0;
            long long gsum = 0;
            for (size_t q = 0; q < ns; ++q) {
                const LaunchRec& r = recs[g.scenes[q]][k];
                gx = std::max(gx, r.grid.x);
                gsum += r.grid.x;
                smem = std::max(smem, r.smem);
                std::memcpy(host.data() + g.table_off[k] + q * r.args.size(), r.args.data(), r.args.size());
            }
            g.kern.push_back(r0[k].kern);
            g.prep.push_back(r0[k].prep);
            if (r0[k].prep) {
                // queue form: a persistent grid over all scenes' items
                const long long ctas = std::min<long long>(gsum, (long long)b->queue_per_sm[r0[k].queue_kind] * n_sm);
                g.grid.push_back(dim3((unsigned)std::max<long long>(ctas, 1), 1, 1));
                ++nq;
            } else {
                g.grid.push_back(dim3(gx, (unsigned)ns, 1));
            }
            g.block.push_back(r0[k].block);
            g.smem.push_back(smem);
            if (smem > 48 * 1024)
                NXD_CUDA(cudaFuncSetAttribute(r0[k].kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        }
        NXD_CUDA(cudaMalloc(&g.table, host.size()));
        NXD_CUDA(cudaMemcpy(g.table, host.data(), host.size(), cudaMemcpyHostToDevice));
        const size_t qstride = ns + 2;   // prefix[ns + 1], counter
        if (nq) NXD_CUDA(cudaMalloc(&g.queue, sizeof(int) * qstride * nq));
        NXD_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        int qi = 0;
        for (size_t k = 0; k < L; ++k) {
            void* tab = (unsigned char*)g.table + g.table_off[k];
            if (g.prep[k]) {
                int nw = (int)ns;
                int* prefix = g.queue + qstride * qi++;
                int* counter = prefix + ns + 1;
                void* pargs[] = {&tab, &nw, &prefix, &counter};
                cudaLaunchKernel(g.prep[k], dim3(1), dim3(kQueuePrepThreads), pargs, 0, b->stream);
                cudaLaunchKernel(g.kern[k], g.grid[k], g.block[k], pargs, g.smem[k], b->stream);
                continue;
            }
            void* args[] = {&tab};
            cudaLaunchKernel(g.kern[k], g.grid[k], g.block[k], args, g.smem[k], b->stream);
        }
        NXD_CUDA(cudaStreamEndCapture(b->stream, &g.graph));
        NXD_CUDA(cudaGraphInstantiate(&g.exec, g.graph, 0));
    }
    b->dts.assign(dts, dts + n);
    return NXD_OK;
}

}  // namespace

extern "C" {

nxd_status nxd_batch_create(const nxd_scene_desc* descs, int32_t n, nxd_batch** out) {
    if (!descs || n <= 0 || !out) return NXD_INVALID_ARGUMENT;
    nxd_batch* b = new (std::nothrow) nxd_batch();
    if (!b) return NXD_INVALID_ARGUMENT;
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) { delete b; return NXD_CUDA_ERROR; }
    for (int i = 0; i < n; ++i) {
        nxd_ctx* c = nullptr;
        const nxd_status st = nxd_create(descs + i, &c);
        if (st != NXD_OK) {
            for (nxd_ctx* x : b->ctx) nxd_destroy(x);
            cudaStreamDestroy(b->stream);
            delete b;
            return st;
        }
        c->stream = b->stream;
        c->newton_grid = 1;   // one CTA per scene in the batched Newton launch
        b->ctx.push_back(c);
    }
    *out = b;
    return NXD_OK;
}

nxd_status nxd_batch_timed_steps(nxd_batch* b, const double* dts, int32_t n_steps, double* ms) {
    if (!b || !dts || n_steps < 1 || !ms) return NXD_INVALID_ARGUMENT;
    cudaEvent_t e0, e1;
    NXD_CUDA(cudaEventCreate(&e0));
    NXD_CUDA(cudaEventCreate(&e1));
    NXD_CUDA(cudaEventRecord(e0, b->stream));
    nxd_status st = NXD_OK;
    for (int k = 0; k < n_steps && st == NXD_OK; ++k) st = nxd_batch_step(b, dts);
    NXD_CUDA(cudaEventRecord(e1, b->stream));
    NXD_CUDA(cudaEventSynchronize(e1));
    float f = 0.0f;
    cudaEventElapsedTime(&f, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = f;
    return st;
}

nxd_status nxd_device_info(int32_t* sm_count, char* name, int32_t name_len) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return NXD_NO_DEVICE;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return NXD_CUDA_ERROR;
    if (sm_count) *sm_count = prop.multiProcessorCount;
    if (name && name_len > 0) {
        std::strncpy(name, prop.name, (size_t)name_len - 1);
        name[name_len - 1] = 0;
    }
    return NXD_OK;
}

nxd_status nxd_batch_set_queue_ctas(nxd_batch* b, int32_t kernel, int32_t ctas_per_sm) {
    if (!b || kernel < 0 || kernel >= kQueueKinds || ctas_per_sm < 1 || ctas_per_sm > 64) return NXD_INVALID_ARGUMENT;
    if (b->queue_per_sm[kernel] != ctas_per_sm) {
        NXD_CUDA(cudaStreamSynchronize(b->stream));
        b->queue_per_sm[kernel] = ctas_per_sm;
        release_groups(b);   // rebuilt at the next step
        b->dts.clear();
    }
    return NXD_OK;
}

void nxd_batch_destroy(nxd_batch* b) {
    if (!b) return;
    cudaStreamSynchronize(b->stream);
    release_groups(b);
    for (cudaStream_t st : b->gstream) cudaStreamDestroy(st);
    for (cudaEvent_t ev : b->gdone) cudaEventDestroy(ev);
    if (b->fork) cudaEventDestroy(b->fork);
    for (nxd_ctx* c : b->ctx) { c->stream = nullptr; nxd_destroy(c); }
    if (b->own_stream) cudaStreamDestroy(b->stream);
    delete b;
}

nxd_status nxd_batch_step(nxd_batch* b, const double* dts) {
    if (!b || !dts) return NXD_INVALID_ARGUMENT;
    for (size_t i = 0; i < b->ctx.size(); ++i)
        if (!(dts[i] > 0.0)) return NXD_INVALID_ARGUMENT;
    bool same = b->dts.size() == b->ctx.size() && !b->groups.empty();
    for (size_t i = 0; same && i < b->ctx.size(); ++i) same = b->dts[i] == dts[i];
    if (!same) {
        NXD_CUDA(cudaStreamSynchronize(b->stream));
        const nxd_status st = build_groups(b, dts);
        if (st != NXD_OK) return st;
    }
    if (b->groups.size() == 1) {
        NXD_CUDA(cudaGraphLaunch(b->groups[0].exec, b->stream));
        return NXD_OK;
    }
    if (!b->fork) NXD_CUDA(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
    while (b->gstream.size() < b->groups.size()) {
        cudaStream_t st;
        cudaEvent_t ev;
        NXD_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        NXD_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        b->gstream.push_back(st);
        b->gdone.push_back(ev);
    }
    NXD_CUDA(cudaEventRecord(b->fork, b->stream));
    for (size_t i = 0; i < b->groups.size(); ++i) {
        NXD_CUDA(cudaStreamWaitEvent(b->gstream[i], b->fork, 0));
        NXD_CUDA(cudaGraphLaunch(b->groups[i].exec, b->gstream[i]));
        NXD_CUDA(cudaEventRecord(b->gdone[i], b->gstream[i]));
        NXD_CUDA(cudaStreamWaitEvent(b->stream, b->gdone[i], 0));
    }
    return NXD_OK;
}

int32_t nxd_batch_groups(nxd_batch* b) { return b ? (int32_t)b->groups.size() : 0; }

nxd_status nxd_batch_set_stream(nxd_batch* b, void* stream) {
    if (!b || !stream) return NXD_INVALID_ARGUMENT;
    NXD_CUDA(cudaStreamSynchronize(b->stream));
    b->stream = (cudaStream_t)stream;
    b->own_stream = false;
    for (nxd_ctx* c : b->ctx) c->stream = b->stream;
    return NXD_OK;
}

nxd_status nxd_batch_get_state(nxd_batch* b, int32_t scene, const nxd_state* o) {
    if (!b || scene < 0 || scene >= (int)b->ctx.size()) return NXD_INVALID_ARGUMENT;
    return nxd_get_state(b->ctx[scene], o);
}

nxd_status nxd_batch_get_diagnostics(nxd_batch* b, int32_t scene, nxd_diagnostics* o) {
    if (!b || scene < 0 || scene >= (int)b->ctx.size()) return NXD_INVALID_ARGUMENT;
    return nxd_get_diagnostics(b->ctx[scene], o);
}

}  // extern "C"
