// geometry.cuh — device kernels for the contact set of one time step:
// body boxes, world vertices, body-pair broad phase, top-32 primitive
// selection, candidate materialisation, the narrow phase of
// detectContacts / detectContactsAtState and the pruned scene minimum distance.
//
// Layout in HBM (SoA per quantity, FP64 / int32):
//   boxes[N*6]      world AABB per body (min xyz, max xyz)
//   wv[nv*3]        world vertices for the pose being tested
//   pairs[P*2]      candidate body pairs, world indices, reference order
//   topk[P*6*32]    selected primitive ids per pair: vA vB eA eB fA fB
//   topn[P*6]       selection sizes min(32, count)
#pragma once

#include "nx_math.cuh"
#include "select.cuh"

namespace nx {

constexpr int kTopK = 32;                 // kMax{Vertices,Edges,Faces}PerBody
constexpr int kMaxRawContacts = 40000;    // IPCSolver.cpp:413
constexpr int kMaxContacts = 2000;        // IPCSolver.cpp:414
constexpr double kPruneBand = 1e-6;       // scene-min-distance exactness band

struct Geo {
    int N;
    const int* voff; const int* foff; const int* eoff;
    const double* verts; const int* faces; const int* edges;
    const double* lmin; const double* lmax;   // local AABB per body [N*3]
    const int* has_mesh;                      // [N]
    const double* md_tol;                     // [N] pruning slack per face body
};

__device__ __forceinline__ Box ld_box(const double* b) { Box r; r.mn = ld3(b); r.mx = ld3(b + 3); return r; }
__device__ __forceinline__ void st_box(double* b, const Box& x) { st3(b, x.mn); st3(b + 3, x.mx); }

// ---------------------------------------------------------------------------
// ContactAssembler::build (ContactAssembler.cpp:124-154): world boxes
// ---------------------------------------------------------------------------
__device__ __forceinline__ void body_boxes_body(const Geo& g, const double* pos, const double* quat, double* boxes) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.N) return;
    const Box b = transform_local_box(ld3(g.lmin + 3 * i), ld3(g.lmax + 3 * i), ld3(pos + 3 * i), ldq(quat + 4 * i));
    st_box(boxes + 6 * i, b);
}
constexpr int kLB_body_boxes = 0;
__global__ void k_body_boxes(const __grid_constant__ Geo g, const double* pos, const double* quat, double* boxes) { body_boxes_body(g, pos, quat, boxes); }

// pose of body i at x: p = x[6i..], q = exp(theta) q_ref ('>' threshold)
__device__ __forceinline__ void pose_at_x_body(int N, const double* x, const double* quat_ref, double* pp, double* pq) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    st3(pp + 3 * i, ld3(x + 6 * i));
    stq(pq + 4 * i, rot_gt(ldq(quat_ref + 4 * i), ld3(x + 6 * i + 3)));
}
constexpr int kLB_pose_at_x = 0;
__global__ void k_pose_at_x(int N, const double* x, const double* quat_ref, double* pp, double* pq) { pose_at_x_body(N, x, quat_ref, pp, pq); }

// world vertex = p + q * v_local (one thread per vertex)
__device__ __forceinline__ void world_vertices_body(const Geo& g, int nv, const int* vbody, const double* pos, const double* quat, double* wv) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nv) return;
    const int b = vbody[v];
    st3(wv + 3 * v, ld3(pos + 3 * b) + qrot(ldq(quat + 4 * b), ld3(g.verts + 3 * v)));
}
constexpr int kLB_world_vertices = 0;
__global__ void k_world_vertices(const __grid_constant__ Geo g, int nv, const int* vbody, const double* pos, const double* quat, double* wv) { world_vertices_body(g, nv, vbody, pos, quat, wv); }

// ---------------------------------------------------------------------------
// Broad phase (ContactAssembler::detectBodyPairs, ContactAssembler.cpp:156-178
// -> IncrementalBVHBroadPhase::detect, BroadPhase.cpp:84-131).  The BVH the
// reference builds never reorders its primitive list (the SAH split count is
// applied to the list in input order, BVH.cpp:336-356), and its stack
// traversal pops the right child first (BVH.cpp:57-90), so for each i the
// overlapping j > i come out in descending j.  The pair set is exactly
// {i<j : inflate(box_i, r) and inflate(box_j, r) overlap (closed)}.
// mode 0: that set; mode 1: additionally aabb_distance(box_i, box_j) <= act
// (buildCandidateSet's filter, ContactAssembler.cpp:240-242); mode 2: the
// scene-min-distance band of the face body j.
// ---------------------------------------------------------------------------
struct PairQuery {
    int mode;
    const double* r_ptr;     // device scalar radius (or null: r_val)
    double r_val;
    double r_scale;          // r = r_scale * (*r_ptr or r_val)
    double act_scale;        // mode 1: act = act_scale * radius
};
__device__ __forceinline__ double pq_radius(const PairQuery& q) {
    return q.r_scale * (q.r_ptr ? *q.r_ptr : q.r_val);
}
__device__ __forceinline__ bool pair_test(const Geo& g, const PairQuery& q, const double* boxes, int i, int j, double r) {
    if (!g.has_mesh[i] || !g.has_mesh[j]) return false;
    const Box bi = ld_box(boxes + 6 * i), bj = ld_box(boxes + 6 * j);
    const double m = dmax(0.0, r);
    if (!box_intersects(box_inflated(bi, m), box_inflated(bj, m))) return false;
    if (q.mode == 1) return !(box_distance(bi, bj) > q.act_scale * (q.r_ptr ? *q.r_ptr : q.r_val));
    if (q.mode == 2) return !(box_distance(bi, bj) > kPruneBand + g.md_tol[j]);
    return true;
}

// one warp per i: count (out == nullptr) or write pairs in descending j
__device__ __forceinline__ void pairs_body(const Geo& g, const PairQuery& q, const double* boxes, int* counts, const int* offsets, int* out, int cap, const int* gate) {
    if (gate && *gate == 0) return;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const double r = pq_radius(q);
    const unsigned lt = (1u << lane) - 1u;
    for (int i = warp; i < g.N; i += nw) {
        int c = 0;
        const int base = out ? offsets[i] : 0;
        for (int top = g.N - 1; top > i; top -= 32) {
            const int j = top - lane;
            const bool f = j > i && pair_test(g, q, boxes, i, j, r);
            const unsigned b = __ballot_sync(0xffffffffu, f);
            if (out && f) {
                const int pos = base + c + __popc(b & lt);
                if (pos < cap) { out[2 * pos] = i; out[2 * pos + 1] = j; }
            }
            c += __popc(b);
        }
        if (!out && lane == 0) counts[i] = c;
    }
}
constexpr int kLB_pairs = 0;
__global__ void k_pairs(const __grid_constant__ Geo g, const __grid_constant__ PairQuery q, const double* boxes, int* counts, const int* offsets, int* out, int cap, const int* gate) { pairs_body(g, q, boxes, counts, offsets, out, cap, gate); }

// Exclusive scan of n ints (single block, 1024 threads); total -> *total.
// n_dev (optional) caps n at a device-side count.  The scan runs only when
// run_if is null or non-zero and skip_if is null or zero; when run_if is zero
// the total is cleared, when skip_if is set nothing is written.
// Exclusive prefix sums of in[0..n) into out (in place allowed) by one CTA;
// returns the total.  Each round, every thread takes kScanItems consecutive
// elements, so a round covers blockDim.x * kScanItems of them with two block
// barriers (the step's pair and hit counts, ~10^4 entries, take one round).
constexpr int kScanItems = 16;
__device__ int block_scan(const int* in, int* out, int n) {
    __shared__ int warp_sums[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int per_round = blockDim.x * kScanItems;
    for (int base = 0; base < n; base += per_round) {
        const int i0 = base + threadIdx.x * kScanItems;
        int v[kScanItems];
        int tsum = 0;
#pragma unroll
        for (int j = 0; j < kScanItems; ++j) {
            v[j] = i0 + j < n ? in[i0 + j] : 0;
            tsum += v[j];
        }
        int x = tsum;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_sums[wid] = x;
        __syncthreads();
        if (wid == 0) {
            int sv = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, sv, o);
                if (lane >= o) sv += y;
            }
            warp_sums[lane] = sv;
        }
        __syncthreads();
        int run = carry + (wid > 0 ? warp_sums[wid - 1] : 0) + x - tsum;
#pragma unroll
        for (int j = 0; j < kScanItems; ++j) {
            if (i0 + j < n) out[i0 + j] = run;
            run += v[j];
        }
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = run;
        __syncthreads();
    }
    const int total = carry;
    __syncthreads();
    return total;
}

__device__ __forceinline__ void scan_body(const int* in, int* out, int n, int* total, const int* run_if, const int* skip_if, const int* n_dev) {
    if (skip_if && *skip_if != 0) return;
    if (run_if && *run_if == 0) { if (threadIdx.x == 0 && total) *total = 0; return; }
    if (n_dev) n = min(n, *n_dev);
    const int t = block_scan(in, out, n);
    if (threadIdx.x == 0 && total) *total = t;
}
constexpr int kLB_scan = 0;
__global__ void k_scan(const int* in, int* out, int n, int* total, const int* run_if, const int* skip_if = nullptr, const int* n_dev = nullptr) { scan_body(in, out, n, total, run_if, skip_if, n_dev); }

// ---------------------------------------------------------------------------
// estimateMinBodyPairDistance (ContactAssembler.cpp:180-212): min over the
// pairs detected with radius r of the un-inflated box distance.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void atomic_min_pos_double(double* addr, double v) {
    // non-negative doubles order like their bit patterns
    atomicMin(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}
__device__ __forceinline__ void min_pair_distance_body(const Geo& g, const PairQuery& q, const double* boxes, double* out) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const double r = pq_radius(q);
    double m = INFINITY;
    for (int i = warp; i < g.N; i += nw)
        for (int j = i + 1 + lane; j < g.N; j += 32)
            if (pair_test(g, q, boxes, i, j, r)) m = dmin(m, box_distance(ld_box(boxes + 6 * i), ld_box(boxes + 6 * j)));
    for (int o = 16; o > 0; o >>= 1) m = dmin(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0 && m < INFINITY) atomic_min_pos_double(out, m);
}
constexpr int kLB_min_pair_distance = 0;
__global__ void k_min_pair_distance(const __grid_constant__ Geo g, const __grid_constant__ PairQuery q, const double* boxes, double* out) { min_pair_distance_body(g, q, boxes, out); }

// ---------------------------------------------------------------------------
// Top-k selection (ContactAssembler.cpp:214-303), lists s = 0 vA, 1 vB, 2 eA,
// 3 eB, 4 fA, 5 fB.  Scores are point-to-box distances of the primitive's
// world vertices to the other body's box.  One warp per (pair, side): the
// side's vertex scores are computed once, and an edge's (face's) score is the
// std::min of its vertices' scores, the same value the per-list evaluation
// gives.  Shared memory per warp: vertex scores, one list's scores, and the
// selection's idx / G / L arrays.
// ---------------------------------------------------------------------------
__host__ __device__ inline size_t topk_warp_bytes(int max_prims, int max_verts) {
    return ((size_t)max_verts * sizeof(double) + (size_t)max_prims * (sizeof(double) + 3 * sizeof(int)) + 31) / 16 * 16;
}
__device__ __forceinline__ void topk_body(const Geo& g, const int* pairs, const int* npairs_ptr, int cap, const double* boxes, const double* wv, int* topk, int* topn, int max_prims, int max_verts) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int wpb = blockDim.x >> 5;
    const int wid = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    unsigned char* base = smem_raw + topk_warp_bytes(max_prims, max_verts) * wid;
    double* vkey = reinterpret_cast<double*>(base);
    double* key = vkey + max_verts;
    int* idx = reinterpret_cast<int*>(key + max_prims);
    const int np = min(*npairs_ptr, cap);
    for (int item = blockIdx.x * wpb + wid; item < np * 2; item += gridDim.x * wpb) {
        const int p = item >> 1, side = item & 1;
        const int a = pairs[2 * p], b = pairs[2 * p + 1];
        const int X = side ? b : a;
        const int Y = side ? a : b;
        const Box other = ld_box(boxes + 6 * Y);
        const int vo = g.voff[X], nv = g.voff[X + 1] - vo;
        for (int e = lane; e < nv; e += 32) vkey[e] = point_box_distance(ld3(wv + 3 * (vo + e)), other);
        __syncwarp();
        for (int list = 0; list < 3; ++list) {
            const double* kk = key;
            int n, s;
            if (list == 0) {
                s = 2 + side;
                const int eo = g.eoff[X];
                n = g.eoff[X + 1] - eo;
                for (int e = lane; e < n; e += 32) {
                    const int* ed = g.edges + 2 * (eo + e);
                    key[e] = dmin(vkey[ed[0]], vkey[ed[1]]);
                }
            } else if (list == 1) {
                s = 4 + side;
                const int fo = g.foff[X];
                n = g.foff[X + 1] - fo;
                for (int e = lane; e < n; e += 32) {
                    const int* f = g.faces + 3 * (fo + e);
                    key[e] = dmin(dmin(vkey[f[0]], vkey[f[1]]), vkey[f[2]]);
                }
            } else {
                s = side;
                n = nv;
                kk = vkey;
            }
            __syncwarp();
            const SelView v{idx, kk, idx + max_prims, idx + 2 * max_prims};
            const int k = min(kTopK, n);
            sel_top_k_warp(v, n, k);
            const size_t out = (size_t)p * 6 + s;
            if (lane < k) topk[out * kTopK + lane] = idx[lane];
            if (lane == 0) topn[out] = k;
            __syncwarp();
        }
    }
}
constexpr int kLB_topk = 0;
__global__ void k_topk(const __grid_constant__ Geo g, const int* pairs, const int* npairs_ptr, int cap, const double* boxes, const double* wv, int* topk, int* topn, int max_prims, int max_verts) { topk_body(g, pairs, npairs_ptr, cap, boxes, wv, topk, topn, max_prims, max_verts); }

// ---------------------------------------------------------------------------
// Candidate item counts per pair and the materialised candidate lists
// (ContactAssembler.cpp:304-341 order).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void item_counts_body(const int* npairs_ptr, int cap, const int* topn, int* nfv, int* nee, int* nvv, int* nev) {
    const int np = min(*npairs_ptr, cap);
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < np; p += gridDim.x * blockDim.x) {
        const int* t = topn + 6 * p;
        nfv[p] = t[4] * t[1] + t[5] * t[0];
        nee[p] = t[2] * t[3];
        nvv[p] = t[0] * t[1];
        if (nev) nev[p] = t[2] * t[1] + t[3] * t[0];
    }
}
constexpr int kLB_item_counts = 0;
__global__ void k_item_counts(const int* npairs_ptr, int cap, const int* topn, int* nfv, int* nee, int* nvv, int* nev) { item_counts_body(npairs_ptr, cap, topn, nfv, nee, nvv, nev); }

struct CandOut {
    int* vv; long long vv_cap;
    int* ev; long long ev_cap;
    int* ee; long long ee_cap;
    int* fv; long long fv_cap;
};
__global__ void k_materialize(Geo g, const int* body_ids, const int* pairs, const int* npairs_ptr, int cap, const int* topk,
                              const int* topn, const int* off_vv, const int* off_ev, const int* off_ee, const int* off_fv,
                              CandOut o) {
    const int np = min(*npairs_ptr, cap);
    for (int p = blockIdx.x; p < np; p += gridDim.x) {
        const int A = pairs[2 * p], B = pairs[2 * p + 1];
        const int idA = body_ids[A], idB = body_ids[B];
        const int* T = topk + (size_t)p * 6 * kTopK;
        const int* n = topn + 6 * p;
        const int* EA = g.edges + 2 * g.eoff[A];
        const int* EB = g.edges + 2 * g.eoff[B];
        for (int t = threadIdx.x; t < n[0] * n[1]; t += blockDim.x) {
            const long long pos = off_vv[p] + t;
            if (pos < o.vv_cap) { int* r = o.vv + 4 * pos; r[0] = idA; r[1] = idB; r[2] = T[t / n[1]]; r[3] = T[kTopK + t % n[1]]; }
        }
        const int ev1 = n[2] * n[1];
        for (int t = threadIdx.x; t < ev1 + n[3] * n[0]; t += blockDim.x) {
            const long long pos = off_ev[p] + t;
            if (pos >= o.ev_cap) continue;
            int* r = o.ev + 5 * pos;
            if (t < ev1) {
                const int e = T[2 * kTopK + t / n[1]];
                r[0] = idA; r[1] = idB; r[2] = EA[2 * e]; r[3] = EA[2 * e + 1]; r[4] = T[kTopK + t % n[1]];
            } else {
                const int u = t - ev1;
                const int e = T[3 * kTopK + u / n[0]];
                r[0] = idB; r[1] = idA; r[2] = EB[2 * e]; r[3] = EB[2 * e + 1]; r[4] = T[u % n[0]];
            }
        }
        for (int t = threadIdx.x; t < n[2] * n[3]; t += blockDim.x) {
            const long long pos = off_ee[p] + t;
            if (pos >= o.ee_cap) continue;
            const int ea = T[2 * kTopK + t / n[3]], eb = T[3 * kTopK + t % n[3]];
            int* r = o.ee + 6 * pos;
            r[0] = idA; r[1] = idB; r[2] = EA[2 * ea]; r[3] = EA[2 * ea + 1]; r[4] = EB[2 * eb]; r[5] = EB[2 * eb + 1];
        }
        const int fv1 = n[4] * n[1];
        for (int t = threadIdx.x; t < fv1 + n[5] * n[0]; t += blockDim.x) {
            const long long pos = off_fv[p] + t;
            if (pos >= o.fv_cap) continue;
            int* r = o.fv + 4 * pos;
            if (t < fv1) { r[0] = idA; r[1] = idB; r[2] = T[4 * kTopK + t / n[1]]; r[3] = T[kTopK + t % n[1]]; }
            else { const int u = t - fv1; r[0] = idB; r[1] = idA; r[2] = T[5 * kTopK + u / n[0]]; r[3] = T[u % n[0]]; }
        }
    }
}

// ---------------------------------------------------------------------------
// Narrow phase (IPCSolver.cpp:32-134 helpers, 394-580 / 582-806)
// ---------------------------------------------------------------------------
struct ContactRec {   // nxd_contact layout
    double point[3];
    double normal[3];
    double distance;
    int body_a, body_b, type, prim_a, prim_b, pad;
};

__device__ __forceinline__ double clamp01(double v) { return (v < 0.0) ? 0.0 : ((1.0 < v) ? 1.0 : v); }

// closestPointsOnSegments (IPCSolver.cpp:32-90) given d1 = q1 - p1,
// a = |d1|^2, d2 = q2 - p2, e = |d2|^2
__device__ __forceinline__ void closest_points_core(V3 p1, V3 d1, double a, V3 p2, V3 d2, double e, V3& c1, V3& c2) {
    const double eps = 1e-12;
    const V3 r = p1 - p2;
    const double f = dot(d2, r);
    double s, t;
    if (a <= eps && e <= eps) { c1 = p1; c2 = p2; return; }
    if (a <= eps) {
        s = 0.0; t = clamp01(f / e);
    } else {
        const double c = dot(d1, r);
        if (e <= eps) {
            t = 0.0; s = clamp01(-c / a);
        } else {
            const double b = dot(d1, d2);
            const double denom = a * e - b * b;
            if (fabs(denom) > eps) s = clamp01((b * f - c * e) / denom);
            else s = 0.0;
            t = (b * s + f) / e;
            if (t < 0.0) { t = 0.0; s = clamp01(-c / a); }
            else if (t > 1.0) { t = 1.0; s = clamp01((b - c) / a); }
        }
    }
    c1 = p1 + d1 * s;
    c2 = p2 + d2 * t;
}
__device__ __forceinline__ void closest_points_on_segments(V3 p1, V3 q1, V3 p2, V3 q2, V3& c1, V3& c2) {
    const V3 d1 = q1 - p1, d2 = q2 - p2;
    closest_points_core(p1, d1, dot(d1, d1), p2, d2, dot(d2, d2), c1, c2);
}
__device__ __forceinline__ V3 safe_normalized(V3 v, V3 fb) {
    const double n = norm(v);
    if (n > 1e-12) return v / n;
    const double fn = norm(fb);
    if (fn > 1e-12) return fb / fn;
    return v3(0, 1, 0);
}
__device__ __forceinline__ bool point_in_triangle(V3 p, V3 a, V3 b, V3 c) {
    const double eps = 1e-8;
    const V3 v0 = b - a, v1 = c - a, v2 = p - a;
    const double d00 = dot(v0, v0), d01 = dot(v0, v1), d11 = dot(v1, v1), d20 = dot(v2, v0), d21 = dot(v2, v1);
    const double denom = d00 * d11 - d01 * d01;
    if (fabs(denom) < 1e-16) return false;
    const double v = (d11 * d20 - d01 * d21) / denom;
    const double w = (d00 * d21 - d01 * d20) / denom;
    const double u = 1.0 - v - w;
    return u >= -eps && v >= -eps && w >= -eps;
}

struct NarrowIn {
    Geo g;
    const int* pairs; const int* npairs_ptr; int cap;
    const int* topk; const int* topn;
    const double* wv;                 // world vertices at the tested pose
    const double* pose_p;             // body positions at the tested pose [N*3]
    const double* dhat_ptr;
    const unsigned long long* allowed;  // sorted (lo world index << 32 | hi) keys of the allowed
    int n_allowed;                      // contact pairs; 0: every pair is allowed
};

__device__ __forceinline__ unsigned long long body_pair_key(int a, int b) {
    const int lo = a < b ? a : b, hi = a < b ? b : a;
    return ((unsigned long long)(unsigned)lo << 32) | (unsigned)hi;
}
// IPCSolver::isContactPairAllowed (IPCSolver.cpp:283-289) by binary search
__device__ __forceinline__ int allowed_index(const unsigned long long* keys, int n, int a, int b) {
    const unsigned long long k = body_pair_key(a, b);
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (keys[mid] < k) lo = mid + 1;
        else hi = mid;
    }
    return lo < n && keys[lo] == k ? lo : -1;
}

// kind 0 = FV, 1 = EE, 2 = VV; item t of pair p.  Returns hit and fills rec.
__device__ bool narrow_item(const NarrowIn& in, int kind, int p, int t, ContactRec* rec) {
    const int A = in.pairs[2 * p], B = in.pairs[2 * p + 1];
    const int* T = in.topk + (size_t)p * 6 * kTopK;
    const int* n = in.topn + 6 * p;
    const double dh = *in.dhat_ptr;
    int ba, bb, type, pa, pb;
    V3 point, normal;
    double dist;
    if (kind == 0) {
        int fb, vb, f, vtx;
        const int fv1 = n[4] * n[1];
        if (t < fv1) { fb = A; vb = B; f = T[4 * kTopK + t / n[1]]; vtx = T[kTopK + t % n[1]]; }
        else { const int u = t - fv1; fb = B; vb = A; f = T[5 * kTopK + u / n[0]]; vtx = T[u % n[0]]; }
        const int* F = in.g.faces + 3 * (in.g.foff[fb] + f);
        const int vo = in.g.voff[fb];
        const V3 v0 = ld3(in.wv + 3 * (vo + F[0])), v1 = ld3(in.wv + 3 * (vo + F[1])), v2 = ld3(in.wv + 3 * (vo + F[2]));
        const V3 pp = ld3(in.wv + 3 * (in.g.voff[vb] + vtx));
        const V3 nn = safe_normalized(cross(v1 - v0, v2 - v0), v3(0, 1, 0));
        const double sd = dot(pp - v0, nn);
        dist = fabs(sd);
        if (dist >= dh) return false;
        const V3 proj = pp - sd * nn;
        if (!point_in_triangle(proj, v0, v1, v2)) return false;
        if (!rec) return true;
        ba = fb; bb = vb; type = 0; pa = f; pb = vtx;
        point = 0.5 * (proj + pp);
        normal = (sd >= 0.0) ? nn : -nn;
    } else if (kind == 1) {
        const int ea = T[2 * kTopK + t / n[3]], eb = T[3 * kTopK + t % n[3]];
        const int* EA = in.g.edges + 2 * (in.g.eoff[A] + ea);
        const int* EB = in.g.edges + 2 * (in.g.eoff[B] + eb);
        const int voA = in.g.voff[A], voB = in.g.voff[B];
        const V3 a0 = ld3(in.wv + 3 * (voA + EA[0])), a1 = ld3(in.wv + 3 * (voA + EA[1]));
        const V3 b0 = ld3(in.wv + 3 * (voB + EB[0])), b1 = ld3(in.wv + 3 * (voB + EB[1]));
        V3 c0, c1;
        closest_points_on_segments(a0, a1, b0, b1, c0, c1);
        const V3 delta = c1 - c0;
        dist = norm(delta);
        if (dist >= dh) return false;
        if (!rec) return true;
        ba = A; bb = B; type = 1; pa = EA[0]; pb = EB[0];
        point = 0.5 * (c0 + c1);
        normal = delta;
    } else {
        const int va = T[t / n[1]], vb = T[kTopK + t % n[1]];
        const V3 a = ld3(in.wv + 3 * (in.g.voff[A] + va)), b = ld3(in.wv + 3 * (in.g.voff[B] + vb));
        const V3 d = b - a;
        dist = norm(d);
        if (dist >= dh) return false;
        if (!rec) return true;
        ba = A; bb = B; type = 0; pa = va; pb = vb;
        point = 0.5 * (a + b);
        normal = d;
    }
    // append_contact (IPCSolver.cpp:431-469 / 651-695)
    const V3 PA = ld3(in.pose_p + 3 * ba), PB = ld3(in.pose_p + 3 * bb);
    V3 nn = safe_normalized(normal, PB - PA);
    if (dot(nn, PB - PA) < 0.0) nn = -nn;
    st3(rec->point, point);
    st3(rec->normal, nn);
    rec->distance = dmax(0.0, dist);
    rec->body_a = ba; rec->body_b = bb; rec->type = type; rec->prim_a = pa; rec->prim_b = pb; rec->pad = 0;
    return true;
}

// ---------------------------------------------------------------------------
// Narrow-phase passes over the implicit candidate grids of each pair.
//
// A pair's items form grids in the order of ContactAssembler.cpp:304-341:
// FV side 0 = faces of A x vertices of B, FV side 1 = faces of B x vertices
// of A, EE = edges of A x edges of B, VV = vertices of A x vertices of B;
// item t = row * ncols + col.  One warp owns a pair.  Each lane keeps one row
// primitive (a face, an A-edge or an A-vertex) in registers and walks the
// columns, whose operands the warp stages in shared memory (SoA) and reads
// as broadcasts.  The hits of column c form one 32-bit ballot (bit = row);
// lane c keeps that word in a register and the warp stores its masks only
// when the pair has hits.  Every decision repeats narrow_item's arithmetic on
// the same operands, so the two always agree.
// ---------------------------------------------------------------------------
constexpr int kMaskWords = 3 * kTopK;   // per pair: FV side 0 | FV side 1 | EE (VV reuses the first 32)
constexpr int kRowsWarps = 4;           // warps per block of k_narrow_rows
constexpr int kEmitWarps = 8;           // warps per block of k_narrow_emit

struct NarrowScratch {
    unsigned* mask;        // [cap * kMaskWords] column hit masks
    int* cnt;              // [2 * cap] hits per pair: FV | EE (VV uses the FV half)
    int* off;              // [2 * cap] exclusive prefixes of cnt, per half
};

struct FaceRegs { V3 v0, e0, e1, nn; double d00, d01, d11, denom; };

__device__ __forceinline__ FaceRegs load_face(const NarrowIn& in, int body, int face) {
    const int* F = in.g.faces + 3 * (in.g.foff[body] + face);
    const int vo = in.g.voff[body];
    FaceRegs f;
    f.v0 = ld3(in.wv + 3 * (vo + F[0]));
    const V3 v1 = ld3(in.wv + 3 * (vo + F[1])), v2 = ld3(in.wv + 3 * (vo + F[2]));
    f.e0 = v1 - f.v0; f.e1 = v2 - f.v0;
    f.nn = safe_normalized(cross(f.e0, f.e1), v3(0, 1, 0));
    f.d00 = dot(f.e0, f.e0); f.d01 = dot(f.e0, f.e1); f.d11 = dot(f.e1, f.e1);
    f.denom = f.d00 * f.d11 - f.d01 * f.d01;
    return f;
}

// FV decision of narrow_item: |plane distance| < dhat and the projection
// passes point_in_triangle (IPCSolver.cpp:107-134).
__device__ __forceinline__ bool fv_hit(const FaceRegs& f, V3 pp, double dh) {
    const double sd = dot(pp - f.v0, f.nn);
    if (fabs(sd) >= dh) return false;
    const V3 proj = pp - sd * f.nn;
    const V3 w2 = proj - f.v0;
    const double d20 = dot(w2, f.e0), d21 = dot(w2, f.e1);
    if (fabs(f.denom) < 1e-16) return false;
    const double v = (f.d11 * d20 - f.d01 * d21) / f.denom;
    const double w = (f.d00 * d21 - f.d01 * d20) / f.denom;
    const double u = 1.0 - v - w;
    return u >= -1e-8 && v >= -1e-8 && w >= -1e-8;
}

struct WarpStage {
    double va[3][kTopK], vb[3][kTopK];                 // selected vertices of A and B
    double b0[3][kTopK], bd[3][kTopK], bmid[3][kTopK]; // selected edges of B: start, direction, midpoint
    double bdd[kTopK], bhalf[kTopK];                   // |direction|^2, half length
};

__device__ __forceinline__ V3 ld_col(const double (&a)[3][kTopK], int c) { return v3(a[0][c], a[1][c], a[2][c]); }
__device__ __forceinline__ void st_col(double (&a)[3][kTopK], int c, V3 v) { a[0][c] = v.x; a[1][c] = v.y; a[2][c] = v.z; }

// Pass 1.  mode 0: FV and EE hit masks and counts; mode 1: the VV fallback.
// Block vb of a grid of vg blocks (blockIdx.x / gridDim.x of a plain launch;
// a work item's chunk of the world's pairs in the batched queue form).
__device__ __forceinline__ void narrow_rows_body(const NarrowIn& in, int mode, const NarrowScratch& s, const int* skip_if,
                                                 int vb, int vg) {
    if (skip_if && *skip_if != 0) return;
    __shared__ WarpStage stage[kRowsWarps];
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    WarpStage& W = stage[threadIdx.x >> 5];
    const int np = min(*in.npairs_ptr, in.cap);
    const double dh = *in.dhat_ptr;
    const int nwarps = vg * kRowsWarps;
    for (int p = vb * kRowsWarps + (threadIdx.x >> 5); p < np; p += nwarps) {
        const int A = in.pairs[2 * p], B = in.pairs[2 * p + 1];
        if (in.n_allowed > 0 && allowed_index(in.allowed, in.n_allowed, A, B) < 0) {
            // detectContacts drops every contact of a pair that is not allowed
            if (lane == 0) { s.cnt[p] = 0; if (mode == 0) s.cnt[in.cap + p] = 0; }
            continue;
        }
        const int* T = in.topk + (size_t)p * 6 * kTopK;
        const int* n = in.topn + 6 * p;
        const int n0 = n[0], n1 = n[1], n2 = n[2], n3 = n[3], n4 = n[4], n5 = n[5];
        const int voA = in.g.voff[A], voB = in.g.voff[B];
        __syncwarp();
        if (lane < n0) st_col(W.va, lane, ld3(in.wv + 3 * (voA + T[lane])));
        if (lane < n1) st_col(W.vb, lane, ld3(in.wv + 3 * (voB + T[kTopK + lane])));
        if (mode == 1) {
            const V3 a = lane < n0 ? ld3(in.wv + 3 * (voA + T[lane])) : v3(0, 0, 0);
            __syncwarp();
            unsigned mv = 0;
            int cv = 0;
            for (int c = 0; c < n1; ++c) {
                const V3 d = ld_col(W.vb, c) - a;
                const unsigned b = __ballot_sync(full, lane < n0 && !(norm(d) >= dh));
                if (lane == c) mv = b;
                cv += __popc(b);
            }
            if (lane == 0) s.cnt[p] = cv;
            if (cv) s.mask[(size_t)p * kMaskWords + lane] = mv;
            continue;
        }
        // edges of B (columns of the EE grid)
        if (lane < n3) {
            const int* E = in.g.edges + 2 * (in.g.eoff[B] + T[3 * kTopK + lane]);
            const V3 b0 = ld3(in.wv + 3 * (voB + E[0])), b1 = ld3(in.wv + 3 * (voB + E[1]));
            const V3 d = b1 - b0;
            st_col(W.b0, lane, b0); st_col(W.bd, lane, d); st_col(W.bmid, lane, 0.5 * (b0 + b1));
            W.bdd[lane] = dot(d, d); W.bhalf[lane] = 0.5 * norm(d);
        }
        int cf = 0, ce = 0;
        unsigned m0 = 0, m1 = 0, m2 = 0;
        // FV side 0: lane = face of A, columns = vertices of B
        {
            const FaceRegs f = lane < n4 ? load_face(in, A, T[4 * kTopK + lane]) : FaceRegs{};
            __syncwarp();
            for (int c = 0; c < n1; ++c) {
                const unsigned b = __ballot_sync(full, lane < n4 && fv_hit(f, ld_col(W.vb, c), dh));
                if (lane == c) m0 = b;
                cf += __popc(b);
            }
        }
        // FV side 1: lane = face of B, columns = vertices of A
        {
            const FaceRegs f = lane < n5 ? load_face(in, B, T[5 * kTopK + lane]) : FaceRegs{};
            for (int c = 0; c < n0; ++c) {
                const unsigned b = __ballot_sync(full, lane < n5 && fv_hit(f, ld_col(W.va, c), dh));
                if (lane == c) m1 = b;
                cf += __popc(b);
            }
        }
        // EE: lane = edge of A, columns = edges of B.  An item whose segments'
        // bounding spheres are farther apart than dhat + 1e-9 cannot pass (the
        // closest points lie on the segments up to rounding far below 1e-9).
        {
            V3 a0 = v3(0, 0, 0), d1 = v3(0, 0, 0), ma = v3(0, 0, 0);
            double aa = 0.0, ha = 0.0;
            if (lane < n2) {
                const int* E = in.g.edges + 2 * (in.g.eoff[A] + T[2 * kTopK + lane]);
                a0 = ld3(in.wv + 3 * (voA + E[0]));
                const V3 a1 = ld3(in.wv + 3 * (voA + E[1]));
                d1 = a1 - a0; aa = dot(d1, d1); ma = 0.5 * (a0 + a1); ha = 0.5 * norm(d1);
            }
            for (int c = 0; c < n3; ++c) {
                bool hit = false;
                if (lane < n2) {
                    const V3 dm = ma - ld_col(W.bmid, c);
                    const double r = dh + 1e-9 + ha + W.bhalf[c];
                    if (!(dot(dm, dm) >= r * r)) {
                        V3 c0, c1;
                        closest_points_core(a0, d1, aa, ld_col(W.b0, c), ld_col(W.bd, c), W.bdd[c], c0, c1);
                        hit = !(norm(c1 - c0) >= dh);
                    }
                }
                const unsigned b = __ballot_sync(full, hit);
                if (lane == c) m2 = b;
                ce += __popc(b);
            }
        }
        if (lane == 0) { s.cnt[p] = cf; s.cnt[in.cap + p] = ce; }
        if (cf + ce) {
            unsigned* M = s.mask + (size_t)p * kMaskWords;
            M[lane] = m0; M[kTopK + lane] = m1; M[2 * kTopK + lane] = m2;
        }
    }
}
constexpr int kLB_narrow_rows = 32 * kRowsWarps;
__global__ void __launch_bounds__(32 * kRowsWarps) k_narrow_rows(const __grid_constant__ NarrowIn in, int mode, const __grid_constant__ NarrowScratch s, const int* skip_if) { narrow_rows_body(in, mode, s, skip_if, blockIdx.x, gridDim.x); }
// work items of one world in the queue form: chunks of kRowsWarps pairs
__device__ __forceinline__ int narrow_rows_items(const NarrowIn& in, int, const NarrowScratch&, const int* skip_if) {
    if (skip_if && *skip_if != 0) return 0;
    return (min(*in.npairs_ptr, in.cap) + kRowsWarps - 1) / kRowsWarps;
}

// Exclusive scan of n ints by one block; returns the total (all threads).
// Prefixes of the hit counts: nseg halves of cap entries each (FV, EE), the
// first *npairs_ptr of each; totals -> tot[0..nseg).
__device__ __forceinline__ void hit_scan_body(const int* cnt, int* off, int cap, const int* npairs_ptr, int nseg, int* tot0, int* tot1, const int* skip_if) {
    if (skip_if && *skip_if != 0) return;
    const int np = min(*npairs_ptr, cap);
    for (int sgm = 0; sgm < nseg; ++sgm) {
        const int t = block_scan(cnt + (size_t)sgm * cap, off + (size_t)sgm * cap, np);
        if (threadIdx.x == 0) *(sgm == 0 ? tot0 : tot1) = t;
    }
}
constexpr int kLB_hit_scan = 0;
__global__ void k_hit_scan(const int* cnt, int* off, int cap, const int* npairs_ptr, int nseg, int* tot0, int* tot1, const int* skip_if) { hit_scan_body(cnt, off, cap, npairs_ptr, nseg, tot0, tot1, skip_if); }

// Pass 2: the hits of each pair in item order, written at their global
// position (FV list, then EE at *ee_base; positions past the raw cap are
// dropped, as append_contact does).  One warp per pair; pairs without hits
// return at once.
__device__ __forceinline__ void emit_grid(const NarrowIn& in, int kind, int p, const unsigned* M, int rows, int cols,
                                          int item_base, int& pos, ContactRec* out) {
    const int lane = threadIdx.x & 31;
    const unsigned w = lane < cols ? M[lane] : 0u;
    int mine = 0;
    for (int c = 0; c < cols; ++c) mine += (__shfl_sync(0xffffffffu, w, c) >> lane) & 1u;
    if (lane >= rows) mine = 0;
    int x = mine;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    const int total = __shfl_sync(0xffffffffu, x, 31);
    int q = pos + x - mine;
    for (int c = 0; c < cols; ++c) {
        const unsigned mc = __shfl_sync(0xffffffffu, w, c);
        if (lane < rows && ((mc >> lane) & 1u)) {
            if (q < kMaxRawContacts) {
                ContactRec r;
                narrow_item(in, kind, p, item_base + lane * cols + c, &r);
                out[q] = r;
            }
            ++q;
        }
    }
    pos += total;
}

__device__ __forceinline__ void narrow_emit_body(const NarrowIn& in, int mode, const NarrowScratch& s, const int* ee_base, ContactRec* out, const int* skip_if,
                                                 int vb, int vg) {
    if (skip_if && *skip_if != 0) return;
    const int np = min(*in.npairs_ptr, in.cap);
    const int nwarps = vg * kEmitWarps;
    for (int p = vb * kEmitWarps + (threadIdx.x >> 5); p < np; p += nwarps) {
        const int* n = in.topn + 6 * p;
        const unsigned* M = s.mask + (size_t)p * kMaskWords;
        if (mode == 1) {
            if (s.cnt[p] == 0) continue;
            int pos = s.off[p];
            if (pos < kMaxRawContacts) emit_grid(in, 2, p, M, n[0], n[1], 0, pos, out);
            continue;
        }
        if (s.cnt[p] > 0) {
            int pos = s.off[p];
            if (pos < kMaxRawContacts) {
                emit_grid(in, 0, p, M, n[4], n[1], 0, pos, out);
                emit_grid(in, 0, p, M + kTopK, n[5], n[0], n[4] * n[1], pos, out);
            }
        }
        if (s.cnt[in.cap + p] > 0) {
            int pos = *ee_base + s.off[in.cap + p];
            if (pos < kMaxRawContacts) emit_grid(in, 1, p, M + 2 * kTopK, n[2], n[3], 0, pos, out);
        }
    }
}
constexpr int kLB_narrow_emit = 32 * kEmitWarps;
__global__ void __launch_bounds__(32 * kEmitWarps) k_narrow_emit(const __grid_constant__ NarrowIn in, int mode, const __grid_constant__ NarrowScratch s, const int* ee_base, ContactRec* out, const int* skip_if) { narrow_emit_body(in, mode, s, ee_base, out, skip_if, blockIdx.x, gridDim.x); }
__device__ __forceinline__ int narrow_emit_items(const NarrowIn& in, int, const NarrowScratch&, const int*, ContactRec*,
                                                 const int* skip_if) {
    if (skip_if && *skip_if != 0) return 0;
    return (min(*in.npairs_ptr, in.cap) + kEmitWarps - 1) / kEmitWarps;
}

// ---------------------------------------------------------------------------
// Scene minimum distance, pruned (computeSceneMinDistance,
// AdaptiveBarrier.h:89-162).  A vertex-face test that passes the barycentric
// check with plane distance d places the vertex within d + md_tol[j] of face
// body j's box (md_tol covers the 1e-6 barycentric slack times the body size
// plus rounding), so only pairs, vertices and faces within kPruneBand +
// md_tol[j] are tested; the minimum is exact whenever it is below kPruneBand.
// ---------------------------------------------------------------------------
__device__ double vertex_face_plane_distance(V3 p, V3 v0, V3 v1, V3 v2) {
    const V3 e1 = v1 - v0, e2 = v2 - v0;
    V3 n = cross(e1, e2);
    const double area = norm(n);
    if (area < 1e-12) return INFINITY;
    n = normalized(n);
    const double dist = fabs(dot(p - v0, n));
    const double M[3][3] = {{e1.x, e2.x, n.x}, {e1.y, e2.y, n.y}, {e1.z, e2.z, n.z}};
#define NX_COF(i, j) (M[((i) + 1) % 3][((j) + 1) % 3] * M[((i) + 2) % 3][((j) + 2) % 3] - \
                      M[((i) + 1) % 3][((j) + 2) % 3] * M[((i) + 2) % 3][((j) + 1) % 3])
    const double det = NX_COF(0, 0) * M[0][0] + NX_COF(1, 0) * M[1][0] + NX_COF(2, 0) * M[2][0];
    const double invdet = 1.0 / det;
    const V3 r = p - v0;
    const double i00 = NX_COF(0, 0) * invdet, i01 = NX_COF(1, 0) * invdet, i02 = NX_COF(2, 0) * invdet;
    const double i10 = NX_COF(0, 1) * invdet, i11 = NX_COF(1, 1) * invdet, i12 = NX_COF(2, 1) * invdet;
#undef NX_COF
    const double c0 = i00 * r.x + i01 * r.y + i02 * r.z;
    const double c1 = i10 * r.x + i11 * r.y + i12 * r.z;
    const double b0 = 1.0 - c0 - c1, b1 = c0, b2 = c1;
    const double bmin = dmin(dmin(b0, b1), b2), bmax = dmax(dmax(b0, b1), b2);
    if (bmin >= -1e-6 && bmax <= 1.0 + 1e-6) return dist;
    return INFINITY;
}

// One warp per pair: lanes test 32 vertices of body i against body j's box at
// a time; each vertex that passes is broadcast and the lanes sweep j's faces.
// The two prune tests and the plane distance are those of the per-(vertex,
// face) formulation, so the minimum over the surviving pairs is the same value.
__device__ __forceinline__ void min_distance_body(const Geo& g, const int* pairs, const int* npairs_ptr, int cap, const double* boxes, const double* wv, double* out, const int* gate) {
    if (gate && *gate == 0) return;
    const unsigned full = 0xffffffffu;
    const int np = min(*npairs_ptr, cap);
    const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    double m = INFINITY;
    for (int p = blockIdx.x * wpb + (threadIdx.x >> 5); p < np; p += gridDim.x * wpb) {
        const int i = pairs[2 * p], j = pairs[2 * p + 1];
        const Box bj = ld_box(boxes + 6 * j);
        const double band = kPruneBand + g.md_tol[j];
        const int vi0 = g.voff[i], nvi = g.voff[i + 1] - vi0;
        const int vj0 = g.voff[j];
        const int fj0 = g.foff[j], nfj = g.foff[j + 1] - fj0;
        for (int v0 = 0; v0 < nvi; v0 += 32) {
            V3 pp = v3(0.0, 0.0, 0.0);
            bool near = false;
            if (v0 + lane < nvi) {
                pp = ld3(wv + 3 * (vi0 + v0 + lane));
                near = !(point_box_distance(pp, bj) > band);
            }
            unsigned live = __ballot_sync(full, near);
            while (live) {
                const int src = __ffs(live) - 1;
                live &= live - 1;
                const V3 q = v3(__shfl_sync(full, pp.x, src), __shfl_sync(full, pp.y, src), __shfl_sync(full, pp.z, src));
                for (int fi = lane; fi < nfj; fi += 32) {
                    const int* F = g.faces + 3 * (fj0 + fi);
                    const V3 a = ld3(wv + 3 * (vj0 + F[0])), b = ld3(wv + 3 * (vj0 + F[1])), c = ld3(wv + 3 * (vj0 + F[2]));
                    Box fb = box_empty();
                    box_expand(fb, a); box_expand(fb, b); box_expand(fb, c);
                    if (point_box_distance(q, fb) > band) continue;
                    m = dmin(m, vertex_face_plane_distance(q, a, b, c));
                }
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) m = dmin(m, __shfl_xor_sync(full, m, o));
    if (lane == 0 && m < INFINITY) atomic_min_pos_double(out, m);
}
constexpr int kLB_min_distance = 0;
__global__ void k_min_distance(const __grid_constant__ Geo g, const int* pairs, const int* npairs_ptr, int cap, const double* boxes, const double* wv, double* out, const int* gate) { min_distance_body(g, pairs, npairs_ptr, cap, boxes, wv, out, gate); }

}  // namespace nx
