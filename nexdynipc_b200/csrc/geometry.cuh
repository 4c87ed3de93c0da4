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
__global__ void k_body_boxes(Geo g, const double* pos, const double* quat, double* boxes) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.N) return;
    const Box b = transform_local_box(ld3(g.lmin + 3 * i), ld3(g.lmax + 3 * i), ld3(pos + 3 * i), ldq(quat + 4 * i));
    st_box(boxes + 6 * i, b);
}

// pose of body i at x: p = x[6i..], q = exp(theta) q_ref ('>' threshold)
__global__ void k_pose_at_x(int N, const double* x, const double* quat_ref, double* pp, double* pq) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    st3(pp + 3 * i, ld3(x + 6 * i));
    stq(pq + 4 * i, rot_gt(ldq(quat_ref + 4 * i), ld3(x + 6 * i + 3)));
}

// world vertex = p + q * v_local (one thread per vertex)
__global__ void k_world_vertices(Geo g, int nv, const int* vbody, const double* pos, const double* quat, double* wv) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nv) return;
    const int b = vbody[v];
    st3(wv + 3 * v, ld3(pos + 3 * b) + qrot(ldq(quat + 4 * b), ld3(g.verts + 3 * v)));
}

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
__global__ void k_pairs(Geo g, PairQuery q, const double* boxes, int* counts, const int* offsets, int* out, int cap,
                        const int* gate) {
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

// Exclusive scan of n ints (single block, 1024 threads); total -> *total.
// n_dev (optional) caps n at a device-side count.  The scan runs only when
// run_if is null or non-zero and skip_if is null or zero; when run_if is zero
// the total is cleared, when skip_if is set nothing is written.
__global__ void k_scan(const int* in, int* out, int n, int* total, const int* run_if, const int* skip_if = nullptr,
                       const int* n_dev = nullptr) {
    if (skip_if && *skip_if != 0) return;
    if (run_if && *run_if == 0) { if (threadIdx.x == 0 && total) *total = 0; return; }
    if (n_dev) n = min(n, *n_dev);
    __shared__ int warp_sums[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int base = 0; base < n; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const int v = i < n ? in[i] : 0;
        int x = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_sums[wid] = x;
        __syncthreads();
        if (wid == 0) {
            int s = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o) s += y;
            }
            warp_sums[lane] = s;
        }
        __syncthreads();
        const int excl = carry + (wid > 0 ? warp_sums[wid - 1] : 0) + x - v;
        if (i < n) out[i] = excl;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

// ---------------------------------------------------------------------------
// estimateMinBodyPairDistance (ContactAssembler.cpp:180-212): min over the
// pairs detected with radius r of the un-inflated box distance.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void atomic_min_pos_double(double* addr, double v) {
    // non-negative doubles order like their bit patterns
    atomicMin(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}
__global__ void k_min_pair_distance(Geo g, PairQuery q, const double* boxes, double* out) {
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

// ---------------------------------------------------------------------------
// Top-k selection (ContactAssembler.cpp:214-303): one warp per (pair, list),
// list s = 0 vA, 1 vB, 2 eA, 3 eB, 4 fA, 5 fB.  Scores are point-to-box
// distances of the primitive's world vertices to the other body's box.
// ---------------------------------------------------------------------------
__global__ void k_topk(Geo g, const int* pairs, const int* npairs_ptr, int cap, const double* boxes, const double* wv,
                       int* topk, int* topn, int max_prims) {
    extern __shared__ unsigned char smem_raw[];
    const int wpb = blockDim.x >> 5;
    const int wid = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const size_t per_warp = ((size_t)max_prims * (sizeof(double) + 3 * sizeof(int)) + 31) / 16 * 16;
    unsigned char* base = smem_raw + per_warp * wid;
    double* key = reinterpret_cast<double*>(base);
    int* idx = reinterpret_cast<int*>(key + max_prims);
    SelView v{idx, key, idx + max_prims, idx + 2 * max_prims};
    const int np = min(*npairs_ptr, cap);
    for (int item = blockIdx.x * wpb + wid; item < np * 6; item += gridDim.x * wpb) {
        const int p = item / 6, s = item % 6;
        const int a = pairs[2 * p], b = pairs[2 * p + 1];
        const int X = (s & 1) ? b : a;
        const int Y = (s & 1) ? a : b;
        const Box other = ld_box(boxes + 6 * Y);
        const int vo = g.voff[X];
        int n;
        if (s < 2) {
            n = g.voff[X + 1] - vo;
            for (int e = lane; e < n; e += 32) key[e] = point_box_distance(ld3(wv + 3 * (vo + e)), other);
        } else if (s < 4) {
            const int eo = g.eoff[X];
            n = g.eoff[X + 1] - eo;
            for (int e = lane; e < n; e += 32) {
                const int* ed = g.edges + 2 * (eo + e);
                key[e] = dmin(point_box_distance(ld3(wv + 3 * (vo + ed[0])), other),
                              point_box_distance(ld3(wv + 3 * (vo + ed[1])), other));
            }
        } else {
            const int fo = g.foff[X];
            n = g.foff[X + 1] - fo;
            for (int e = lane; e < n; e += 32) {
                const int* f = g.faces + 3 * (fo + e);
                const double d0 = point_box_distance(ld3(wv + 3 * (vo + f[0])), other);
                const double d1 = point_box_distance(ld3(wv + 3 * (vo + f[1])), other);
                const double d2 = point_box_distance(ld3(wv + 3 * (vo + f[2])), other);
                key[e] = dmin(dmin(d0, d1), d2);
            }
        }
        __syncwarp();
        const int k = min(kTopK, n);
        sel_top_k_warp(v, n, k);
        if (lane < k) topk[(size_t)item * kTopK + lane] = idx[lane];
        if (lane == 0) topn[item] = k;
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Candidate item counts per pair and the materialised candidate lists
// (ContactAssembler.cpp:304-341 order).
// ---------------------------------------------------------------------------
__global__ void k_item_counts(const int* npairs_ptr, int cap, const int* topn, int* nfv, int* nee, int* nvv, int* nev) {
    const int np = min(*npairs_ptr, cap);
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < np; p += gridDim.x * blockDim.x) {
        const int* t = topn + 6 * p;
        nfv[p] = t[4] * t[1] + t[5] * t[0];
        nee[p] = t[2] * t[3];
        nvv[p] = t[0] * t[1];
        if (nev) nev[p] = t[2] * t[1] + t[3] * t[0];
    }
}

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
};

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

// Pass 1: hit flags per item and hit counts per pair.  One block per pair.
__global__ void k_narrow_count(NarrowIn in, int kind, const int* item_off, unsigned char* flags, int* hit_cnt,
                               const int* gate_zero) {
    if (gate_zero && *gate_zero != 0) return;
    const int np = min(*in.npairs_ptr, in.cap);
    __shared__ int red[32];
    for (int p = blockIdx.x; p < np; p += gridDim.x) {
        const int* n = in.topn + 6 * p;
        const int cnt = kind == 0 ? n[4] * n[1] + n[5] * n[0] : (kind == 1 ? n[2] * n[3] : n[0] * n[1]);
        const int off = item_off[p];
        int h = 0;
        for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
            const bool hit = narrow_item(in, kind, p, t, nullptr);
            flags[off + t] = hit ? 1 : 0;
            h += hit ? 1 : 0;
        }
        for (int o = 16; o > 0; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = h;
        __syncthreads();
        if (threadIdx.x == 0) {
            int s = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
            hit_cnt[p] = s;
        }
        __syncthreads();
    }
}

// Pass 2: write hits in item order at base + hit_off[p] (positions past the
// raw cap are dropped, as append_contact does).
__global__ void k_narrow_write(NarrowIn in, int kind, const int* item_off, const unsigned char* flags, const int* hit_off,
                               const int* base_ptr, ContactRec* out, const int* gate_zero) {
    if (gate_zero && *gate_zero != 0) return;
    const int np = min(*in.npairs_ptr, in.cap);
    __shared__ int wsum[32];
    __shared__ int carry;
    const int base = base_ptr ? *base_ptr : 0;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int p = blockIdx.x; p < np; p += gridDim.x) {
        const int* n = in.topn + 6 * p;
        const int cnt = kind == 0 ? n[4] * n[1] + n[5] * n[0] : (kind == 1 ? n[2] * n[3] : n[0] * n[1]);
        const int off = item_off[p];
        if (threadIdx.x == 0) carry = base + hit_off[p];
        __syncthreads();
        for (int b0 = 0; b0 < cnt; b0 += blockDim.x) {
            const int t = b0 + threadIdx.x;
            const int f = t < cnt ? flags[off + t] : 0;
            const unsigned bal = __ballot_sync(0xffffffffu, f);
            if (lane == 0) wsum[wid] = __popc(bal);
            __syncthreads();
            int pre = 0;
            for (int w = 0; w < wid; ++w) pre += wsum[w];
            const int pos = carry + pre + __popc(bal & ((1u << lane) - 1u));
            if (f && pos < kMaxRawContacts) {
                ContactRec r;
                narrow_item(in, kind, p, t, &r);
                out[pos] = r;
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                int tot = 0;
                for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += wsum[w];
                carry += tot;
            }
            __syncthreads();
        }
    }
}

// Pass 1 for FV and EE with the pair's selected primitives staged in shared
// memory: per face its first vertex, edge vectors, unit normal and the
// barycentric Gram terms; per edge its start, direction, |d|^2, midpoint and
// half length; per vertex its position.  Each item then repeats only the
// per-item arithmetic of narrow_item, on the same operands, so its decision
// equals narrow_item's.  An EE item whose segments' bounding spheres are
// farther apart than dhat + 1e-9 cannot pass (the closest-point pair lies on
// the segments up to rounding far below 1e-9) and is rejected first.
constexpr int kFaceStage = 16, kEdgeStage = 12;
__global__ void __launch_bounds__(256) k_narrow_count_staged(NarrowIn in, int kind, const int* item_off, unsigned char* flags,
                                                             int* hit_cnt, const int* gate_zero) {
    if (gate_zero && *gate_zero != 0) return;
    __shared__ double prim[2][kTopK][kFaceStage];
    __shared__ double vtx[2][kTopK][3];
    __shared__ int red[8];
    const int np = min(*in.npairs_ptr, in.cap);
    const double dh = *in.dhat_ptr;
    for (int p = blockIdx.x; p < np; p += gridDim.x) {
        const int AB[2] = {in.pairs[2 * p], in.pairs[2 * p + 1]};
        const int* T = in.topk + (size_t)p * 6 * kTopK;
        const int* n = in.topn + 6 * p;
        const int t0 = threadIdx.x;
        if (t0 < 64) {
            const int side = t0 >> 5, k = t0 & 31, body = AB[side];
            const int vo = in.g.voff[body];
            double* P = prim[side][k];
            if (kind == 0 && k < n[4 + side]) {
                const int* F = in.g.faces + 3 * (in.g.foff[body] + T[(4 + side) * kTopK + k]);
                const V3 v0 = ld3(in.wv + 3 * (vo + F[0])), v1 = ld3(in.wv + 3 * (vo + F[1])), v2 = ld3(in.wv + 3 * (vo + F[2]));
                const V3 e0 = v1 - v0, e1 = v2 - v0;
                const V3 nn = safe_normalized(cross(e0, e1), v3(0, 1, 0));
                const double d00 = dot(e0, e0), d01 = dot(e0, e1), d11 = dot(e1, e1);
                st3(P, v0); st3(P + 3, e0); st3(P + 6, e1); st3(P + 9, nn);
                P[12] = d00; P[13] = d01; P[14] = d11; P[15] = d00 * d11 - d01 * d01;
            } else if (kind == 1 && k < n[2 + side]) {
                const int* E = in.g.edges + 2 * (in.g.eoff[body] + T[(2 + side) * kTopK + k]);
                const V3 a0 = ld3(in.wv + 3 * (vo + E[0])), a1 = ld3(in.wv + 3 * (vo + E[1]));
                const V3 d = a1 - a0;
                st3(P, a0); st3(P + 3, d); P[6] = dot(d, d);
                st3(P + 7, 0.5 * (a0 + a1)); P[10] = 0.5 * norm(d);
            }
        } else if (t0 < 128 && kind == 0) {
            const int side = (t0 - 64) >> 5, k = t0 & 31, body = AB[side];
            if (k < n[side]) st3(vtx[side][k], ld3(in.wv + 3 * (in.g.voff[body] + T[side * kTopK + k])));
        }
        __syncthreads();
        const int cnt = kind == 0 ? n[4] * n[1] + n[5] * n[0] : n[2] * n[3];
        const int fv1 = n[4] * n[1];
        const int off = item_off[p];
        int h = 0;
        for (int t = t0; t < cnt; t += blockDim.x) {
            bool hit = false;
            if (kind == 0) {
                int fs, fi, vs_, vi;
                if (t < fv1) { fs = 0; fi = t / n[1]; vs_ = 1; vi = t % n[1]; }
                else { const int u = t - fv1; fs = 1; fi = u / n[0]; vs_ = 0; vi = u % n[0]; }
                const double* P = prim[fs][fi];
                const V3 a = ld3(P), nn = ld3(P + 9);
                const V3 pp = ld3(vtx[vs_][vi]);
                const double sd = dot(pp - a, nn);
                if (!(fabs(sd) >= dh)) {
                    // point_in_triangle(proj, v0, v1, v2) (IPCSolver.cpp:107-134)
                    const V3 proj = pp - sd * nn;
                    const V3 v2 = proj - a;
                    const double d20 = dot(v2, ld3(P + 3)), d21 = dot(v2, ld3(P + 6));
                    const double d00 = P[12], d01 = P[13], d11 = P[14], denom = P[15];
                    if (!(fabs(denom) < 1e-16)) {
                        const double v = (d11 * d20 - d01 * d21) / denom;
                        const double w = (d00 * d21 - d01 * d20) / denom;
                        const double u = 1.0 - v - w;
                        hit = u >= -1e-8 && v >= -1e-8 && w >= -1e-8;
                    }
                }
            } else {
                const double* EA = prim[0][t / n[3]];
                const double* EB = prim[1][t % n[3]];
                const double lb = norm(ld3(EA + 7) - ld3(EB + 7)) - EA[10] - EB[10];
                if (!(lb >= dh + 1e-9)) {
                    V3 c0, c1;
                    closest_points_core(ld3(EA), ld3(EA + 3), EA[6], ld3(EB), ld3(EB + 3), EB[6], c0, c1);
                    hit = !(norm(c1 - c0) >= dh);
                }
            }
            flags[off + t] = hit ? 1 : 0;
            h += hit ? 1 : 0;
        }
        for (int o = 16; o > 0; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
        if ((t0 & 31) == 0) red[t0 >> 5] = h;
        __syncthreads();
        if (t0 == 0) {
            int sum = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) sum += red[w];
            hit_cnt[p] = sum;
        }
        __syncthreads();
    }
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

__global__ void k_min_distance(Geo g, const int* pairs, const int* npairs_ptr, int cap, const double* boxes,
                               const double* wv, double* out, const int* gate) {
    if (gate && *gate == 0) return;
    const int np = min(*npairs_ptr, cap);
    double m = INFINITY;
    for (int p = blockIdx.x; p < np; p += gridDim.x) {
        const int i = pairs[2 * p], j = pairs[2 * p + 1];
        const Box bj = ld_box(boxes + 6 * j);
        const double band = kPruneBand + g.md_tol[j];
        const int vi0 = g.voff[i], nvi = g.voff[i + 1] - vi0;
        const int vj0 = g.voff[j];
        const int fj0 = g.foff[j], nfj = g.foff[j + 1] - fj0;
        for (int w = threadIdx.x; w < nvi * nfj; w += blockDim.x) {
            const int vi = w / nfj, fi = w % nfj;
            const V3 pp = ld3(wv + 3 * (vi0 + vi));
            if (point_box_distance(pp, bj) > band) continue;
            const int* F = g.faces + 3 * (fj0 + fi);
            const V3 a = ld3(wv + 3 * (vj0 + F[0])), b = ld3(wv + 3 * (vj0 + F[1])), c = ld3(wv + 3 * (vj0 + F[2]));
            Box fb = box_empty();
            box_expand(fb, a); box_expand(fb, b); box_expand(fb, c);
            if (point_box_distance(pp, fb) > band) continue;
            m = dmin(m, vertex_face_plane_distance(pp, a, b, c));
        }
    }
    for (int o = 16; o > 0; o >>= 1) m = dmin(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m < INFINITY) atomic_min_pos_double(out, m);
}

}  // namespace nx
