// ipc.cuh — device side of the primitive-level contact model (full IPC,
// "Mode I"): a linear BVH over dhat-inflated triangle / edge boxes, rebuilt
// from Morton codes for every evaluation state, stack traversal that emits
// the compacted point-triangle and edge-edge candidate lists, the per-pair
// barrier with PSD-projected Hessians chained to 6x6 body blocks (segment
// reduction into BSR), and additive CCD with a block min-reduce.
//
// HBM layout (per context, grown on demand):
//   wq[nv*3], wq1[nv*3]      world vertices at x and at x + dx
//   leaf boxes [n*6]          face / edge boxes, inflated (min xyz, max xyz)
//   keys / ids [n]            (Morton << 32 | index), sorted by a stable LSD
//                             radix sort on the Morton bits
//   nodes: child[2(n-1)], parent[2n-1], box[(2n-1)*6], flags[n-1]
//   pairs pt[n_pt*2] (vertex, face), ee[n_ee*2] (edge i < edge j)
//   per active pair: energy, chained gradient (12), up to 5 (lambda, z[12])
#pragma once

#include "geometry.cuh"
#include "ipc_pair.h"

namespace nx {

// ---------------------------------------------------------------------------
// Stable LSD radix sort of (64-bit key, int value) pairs on key bits
// [lo, hi), 8 bits per pass.  A block sorts a tile of kRsTile items: digit
// histogram, a global digit-major exclusive scan, then a stable scatter
// (rounds of 256 items in tile order; ranks inside a warp from
// __match_any_sync, across warps from per-round digit counts).
// ---------------------------------------------------------------------------
constexpr int kRsThreads = 256;
constexpr int kRsRounds = 16;
constexpr int kRsTile = kRsThreads * kRsRounds;

__global__ void __launch_bounds__(kRsThreads) k_rs_hist(const unsigned long long* keys, int n, int shift, int* hist, int nblocks) {
    __shared__ int h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int base = blockIdx.x * kRsTile;
    for (int r = 0; r < kRsRounds; ++r) {
        const int i = base + r * kRsThreads + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & 0xFF], 1);
    }
    __syncthreads();
    hist[threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

__global__ void k_rs_scan(int* hist, int n) { block_scan(hist, hist, n); }

__global__ void __launch_bounds__(kRsThreads) k_rs_scatter(const unsigned long long* kin, const int* vin, unsigned long long* kout,
                                                           int* vout, int n, int shift, const int* hist, int nblocks) {
    __shared__ int run[256];
    __shared__ int wcnt[kRsThreads / 32][256];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    run[threadIdx.x] = hist[threadIdx.x * nblocks + blockIdx.x];
    for (int k = 0; k < kRsThreads / 32; ++k) wcnt[k][threadIdx.x] = 0;
    __syncthreads();
    const int base = blockIdx.x * kRsTile;
    for (int r = 0; r < kRsRounds; ++r) {
        const int i = base + r * kRsThreads + threadIdx.x;
        const bool ok = i < n;
        const unsigned long long key = ok ? kin[i] : 0ull;
        const int d = ok ? (int)((key >> shift) & 0xFF) : 256 + lane;   // idle lanes never match
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int rank = __popc(peers & ((1u << lane) - 1u));
        const int leader = __ffs(peers) - 1;
        if (ok && lane == leader) wcnt[w][d] = __popc(peers);
        __syncthreads();
        if (ok) {
            int pos = run[d] + rank;
            for (int k = 0; k < w; ++k) pos += wcnt[k][d];
            kout[pos] = key;
            vout[pos] = vin[i];
        }
        __syncthreads();
        // advance the running offsets; clear the counts of this round
        int add = 0;
        for (int k = 0; k < kRsThreads / 32; ++k) { add += wcnt[k][threadIdx.x]; wcnt[k][threadIdx.x] = 0; }
        run[threadIdx.x] += add;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Boxes
// ---------------------------------------------------------------------------
struct PrimGeo {
    int nv, nf, ne;
    const int* vbody;          // [nv]
    const int* fbody;          // [nf]
    const int* ebody;          // [ne]
    const int* fvert;          // [nf*3] global vertex ids
    const int* evert;          // [ne*2] global vertex ids
};

__device__ __forceinline__ void box_of(const double* w0, const double* w1, const int* vid, int nvid, double infl, double* out) {
    V3 mn = ld3(w0 + 3 * vid[0]), mx = mn;
    for (int k = 0; k < nvid; ++k) {
        const V3 a = ld3(w0 + 3 * vid[k]);
        mn = cwmin(mn, a); mx = cwmax(mx, a);
        if (w1) { const V3 b = ld3(w1 + 3 * vid[k]); mn = cwmin(mn, b); mx = cwmax(mx, b); }
    }
    const V3 e = v3(infl, infl, infl);
    st3(out, mn - e);
    st3(out + 3, mx + e);
}

// kind 0: face leaves, 1: edge leaves, 2: vertex queries, 3: edge queries.
// pad (swept boxes of the rigid arcs, per body; may be null) widens each box
// by its body's arc bound (ipc::arc_box_pad).
__global__ void k_ipc_boxes(PrimGeo pg, int kind, const double* w0, const double* w1, double infl, double* out,
                            const double* pad = nullptr) {
    const int n = kind == 0 ? pg.nf : (kind == 2 ? pg.nv : pg.ne);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int b = kind == 0 ? pg.fbody[i] : (kind == 2 ? pg.vbody[i] : pg.ebody[i]);
        const double e = pad ? infl + pad[b] : infl;
        if (kind == 0) box_of(w0, w1, pg.fvert + 3 * i, 3, e, out + 6 * i);
        else if (kind == 2) box_of(w0, w1, &i, 1, e, out + 6 * i);
        else box_of(w0, w1, pg.evert + 2 * i, 2, e, out + 6 * i);
    }
}

// the largest |v| over each body's local vertices (0 for a meshless body)
__global__ void k_body_rmax(Geo g, double* rmax) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < g.N; b += gridDim.x * blockDim.x) {
        double r = 0.0;
        for (int v = g.voff[b]; v < g.voff[b + 1]; ++v) r = dmax(r, norm(ld3(g.verts + 3 * v)));
        rmax[b] = r;
    }
}
// per body the arc pad of the swept boxes along dx
__global__ void k_arc_pad(int N, const double* dx, const double* rmax, double* pad) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < N; b += gridDim.x * blockDim.x)
        pad[b] = ipc::arc_box_pad(ld3(dx + 6 * b + 3), rmax[b]);
}

// Global primitive topology from the body-local meshes: one thread per body.
__global__ void k_prim_topology(Geo g, int* fbody, int* fvert, int* ebody, int* evert) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < g.N; b += gridDim.x * blockDim.x) {
        const int vo = g.voff[b];
        for (int f = g.foff[b]; f < g.foff[b + 1]; ++f) {
            fbody[f] = b;
            for (int k = 0; k < 3; ++k) fvert[3 * f + k] = vo + g.faces[3 * f + k];
        }
        for (int e = g.eoff[b]; e < g.eoff[b + 1]; ++e) {
            ebody[e] = b;
            for (int k = 0; k < 2; ++k) evert[2 * e + k] = vo + g.edges[2 * e + k];
        }
    }
}

__global__ void k_axpy_vec(const double* x, const double* dx, int n, double* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = x[i] + dx[i];
}

// full-IPC time step helpers: out = x + alpha dx; g = gr + s gb and its
// negation; elementwise product; row-wise concatenation of two BSR matrices
// (the second scaled by s), rows of the first before the second's
__global__ void k_axpy_alpha(const double* x, const double* dx, double alpha, int n, double* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = x[i] + alpha * dx[i];
}
__global__ void k_grad_combine(const double* gr, const double* gb, double s, int n, double* g, double* neg) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double v = gr[i] + s * gb[i];
        g[i] = v;
        neg[i] = -v;
    }
}
__global__ void k_mul_vec(const double* a, const double* b, int n, double* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = a[i] * b[i];
}
__global__ void k_bsr_concat(int N, const int* rpa, const int* cia, const double* va, const int* rpb, const int* cib,
                             const double* vb, double s, const int* rpm, int* cim, double* vm) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    int o = rpm[i];
    for (int k = rpa[i]; k < rpa[i + 1]; ++k, ++o) {
        cim[o] = cia[k];
        for (int e = 0; e < 36; ++e) vm[36LL * o + e] = va[36LL * k + e];
    }
    if (!rpb) return;
    for (int k = rpb[i]; k < rpb[i + 1]; ++k, ++o) {
        cim[o] = cib[k];
        for (int e = 0; e < 36; ++e) vm[36LL * o + e] = vb[36LL * k + e] * s;
    }
}

// Exclusive scan of n ints over many CTAs (the candidate counts, active
// flags and segment flags of the full-IPC path reach 10^5 entries, where
// one CTA's rounds cost ~50 us): per tile of kScanTile entries its sum,
// one CTA scans the tile sums (the total with them), then each tile is
// scanned by block_scan and offset.  Integer sums: the same result as k_scan.
constexpr int kScanTileThreads = 256;
constexpr int kScanTile = kScanTileThreads * kScanItems;
__global__ void __launch_bounds__(kScanTileThreads) k_scan_tile_sums(const int* in, int n, int* sums) {
    __shared__ int ws[kScanTileThreads / 32];
    const int base = blockIdx.x * kScanTile, end = min(n, base + kScanTile);
    int v = 0;
    for (int i = base + threadIdx.x; i < end; i += kScanTileThreads) v += in[i];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < kScanTileThreads / 32; ++w) t += ws[w];
        sums[blockIdx.x] = t;
    }
}
__global__ void k_scan_sums(int* sums, int nt, int* total) {
    const int t = block_scan(sums, sums, nt);
    if (threadIdx.x == 0 && total) *total = t;
}
__global__ void __launch_bounds__(kScanTileThreads) k_scan_tiles(const int* in, int* out, int n, const int* offs) {
    const int base = blockIdx.x * kScanTile, m = min(kScanTile, n - base);
    block_scan(in + base, out + base, m);
    __syncthreads();
    const int o = offs[blockIdx.x];
    for (int i = threadIdx.x; i < m; i += kScanTileThreads) out[base + i] += o;
}

// Each query's slice of (query, primitive) pairs, [off[q], off[q] + cnt[q]),
// sorted by primitive in place (the primitives of a slice are distinct).
// Each warp takes 32 consecutive queries: a slice of at most kSliceSortMax
// is sorted by its lane (insertion), and the warp then sorts its longer
// slices one after another together (bitonic network over the slice
// padded to a power of two in the warp's shared row).  Used while no slice
// is longer than kLongSliceMax.
constexpr int kSliceSortMax = 64;
constexpr int kLongSliceMax = 2048;
constexpr int kQueryBuf = 16;     // hits kept per query by k_traverse's count pass
constexpr int kSliceSortThreads = 128;
__global__ void __launch_bounds__(kSliceSortThreads) k_sort_query_slices(int* pairs, const int* off, const int* cnt, int nq) {
    __shared__ int row[kSliceSortThreads / 32][kLongSliceMax];
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    int* sh = row[threadIdx.x >> 5];
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long base = (long long)blockIdx.x * blockDim.x + threadIdx.x - lane; base < nq; base += stride) {
        const int q = (int)base + lane;
        const int m = q < nq ? cnt[q] : 0;
        if (m <= kSliceSortMax) {
            int* p = pairs + 2 * (size_t)(q < nq ? off[q] : 0) + 1;    // primitives at stride 2
            for (int i = 1; i < m; ++i) {
                const int v = p[2 * i];
                int j = i - 1;
                while (j >= 0 && p[2 * j] > v) { p[2 * (j + 1)] = p[2 * j]; --j; }
                p[2 * (j + 1)] = v;
            }
        }
        unsigned longer = __ballot_sync(full, m > kSliceSortMax);
        while (longer) {
            const int src = __ffs(longer) - 1;
            longer &= longer - 1;
            const int mm = __shfl_sync(full, m, src);
            int* p = pairs + 2 * (size_t)off[(int)base + src] + 1;
            int P = 2 * kSliceSortMax;
            while (P < mm) P <<= 1;
            for (int i = lane; i < P; i += 32) sh[i] = i < mm ? p[2 * i] : 0x7fffffff;
            __syncwarp();
            for (int k = 2; k <= P; k <<= 1)
                for (int j = k >> 1; j > 0; j >>= 1) {
                    for (int i = lane; i < P; i += 32) {
                        const int l = i ^ j;
                        if (l > i) {
                            const int x = sh[i], y = sh[l];
                            if ((i & k) == 0 ? x > y : x < y) { sh[i] = y; sh[l] = x; }
                        }
                    }
                    __syncwarp();
                }
            for (int i = lane; i < mm; i += 32) p[2 * i] = sh[i];
            __syncwarp();
        }
    }
}

// Each query's hits from its qbuf row, sorted by primitive (insertion, in
// registers), written as (query, primitive) pairs at off[q].  With `guard`
// (the trial path) nothing is written while a query overflowed its row
// (guard[0] or guard[1] set) or the list would pass `cap` pairs.
__global__ void k_copy_slices(const int* qbuf, const int* cnt, const int* off, int* out, int nq, const int* guard,
                              long long cap) {
    if (guard && (guard[0] | guard[1])) return;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x) {
        const int m = cnt[q];
        if (m == 0 || off[q] + (long long)m > cap) continue;
        int h[kQueryBuf];
#pragma unroll
        for (int i = 0; i < kQueryBuf; ++i) h[i] = i < m ? qbuf[(size_t)kQueryBuf * q + i] : 0x7fffffff;
        // insertion sort over the fixed-size row (the padding sorts last)
#pragma unroll
        for (int i = 1; i < kQueryBuf; ++i) {
#pragma unroll
            for (int j = i; j > 0; --j) {
                const int a = h[j - 1], b = h[j];
                h[j - 1] = a < b ? a : b;
                h[j] = a < b ? b : a;
            }
        }
        int* dst = out + 2 * (size_t)off[q];
        for (int i = 0; i < m; ++i) { dst[2 * i] = q; dst[2 * i + 1] = h[i]; }
    }
}

// pair (q, prim) <-> sort key (q << pbits) | prim
__global__ void k_pair_keys(const int* pairs, int n, int pbits, unsigned long long* key, int* val) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        key[i] = ((unsigned long long)(unsigned)pairs[2 * i] << pbits) | (unsigned)pairs[2 * i + 1];
        val[i] = i;
    }
}
__global__ void k_pair_from_keys(const unsigned long long* key, int n, int pbits, int* pairs) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        pairs[2 * i] = (int)(key[i] >> pbits);
        pairs[2 * i + 1] = (int)(key[i] & ((1ull << pbits) - 1ull));
    }
}

// list[pos[i]] = i for every flagged i (pos = exclusive scan of flag)
__global__ void k_compact(const int* flag, const int* pos, int n, int* list) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (flag[i]) list[pos[i]] = i;
}

// Scene bounds of the leaf-box centroids (one block, fixed order).
__global__ void k_centroid_bounds(const double* box, int n, double* out6) {
    __shared__ double sm[6][32];
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        for (int a = 0; a < 3; ++a) {
            const double c = 0.5 * (box[6 * i + a] + box[6 * i + 3 + a]);
            lo[a] = dmin(lo[a], c); hi[a] = dmax(hi[a], c);
        }
    for (int a = 0; a < 3; ++a)
        for (int o = 16; o > 0; o >>= 1) {
            lo[a] = dmin(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
            hi[a] = dmax(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
        }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
    if (l == 0) for (int a = 0; a < 3; ++a) { sm[a][w] = lo[a]; sm[3 + a][w] = hi[a]; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int a = 0; a < 3; ++a) {
            double L = INFINITY, H = -INFINITY;
            for (int k = 0; k < nw; ++k) { L = dmin(L, sm[a][k]); H = dmax(H, sm[3 + a][k]); }
            out6[a] = L; out6[3 + a] = H;
        }
    }
}

__device__ __forceinline__ unsigned expand_bits10(unsigned v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

// key = (30-bit Morton code of the box centroid) << 32 | leaf index
__global__ void k_morton(const double* box, int n, const double* bounds, unsigned long long* keys, int* ids) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        unsigned q[3];
        for (int a = 0; a < 3; ++a) {
            const double ext = bounds[3 + a] - bounds[a];
            const double c = 0.5 * (box[6 * i + a] + box[6 * i + 3 + a]);
            double u = ext > 0.0 ? (c - bounds[a]) / ext : 0.0;
            u = u < 0.0 ? 0.0 : (u > 1.0 ? 1.0 : u);
            unsigned v = (unsigned)(u * 1023.0);
            q[a] = v > 1023u ? 1023u : v;
        }
        const unsigned m = (expand_bits10(q[0]) << 2) | (expand_bits10(q[1]) << 1) | expand_bits10(q[2]);
        keys[i] = ((unsigned long long)m << 32) | (unsigned)i;
        ids[i] = i;
    }
}

// Karras (2012) hierarchy over sorted unique keys: internal node i spans a
// key range that starts or ends at i; its split is the highest differing bit.
// Children >= 0 are internal nodes, ~leaf for leaves (leaf slot in sorted order).
__device__ __forceinline__ int kdelta(const unsigned long long* k, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    return __clzll(k[i] ^ k[j]);
}

__global__ void k_karras(const unsigned long long* k, int n, int* child, int* parent, int2* rng) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n - 1; i += gridDim.x * blockDim.x) {
        const int d = (kdelta(k, n, i, i + 1) - kdelta(k, n, i, i - 1)) >= 0 ? 1 : -1;
        const int dmin_ = kdelta(k, n, i, i - d);
        int lmax = 2;
        while (lmax < 2 * n && kdelta(k, n, i, i + lmax * d) > dmin_) lmax <<= 1;
        int l = 0;
        for (int t = lmax >> 1; t >= 1; t >>= 1)
            if (kdelta(k, n, i, i + (l + t) * d) > dmin_) l += t;
        const int j = i + l * d;
        const int dnode = kdelta(k, n, i, j);
        int s = 0, t = l;
        while (t > 1) {
            t = (t + 1) >> 1;
            if (kdelta(k, n, i, i + (s + t) * d) > dnode) s += t;
        }
        const int gamma = i + s * d + (d < 0 ? -1 : 0);
        const int lo = i < j ? i : j, hi = i < j ? j : i;
        const int left = lo == gamma ? ~gamma : gamma;
        const int right = hi == gamma + 1 ? ~(gamma + 1) : gamma + 1;
        child[2 * i] = left;
        child[2 * i + 1] = right;
        rng[i] = make_int2(lo, hi);
        parent[left >= 0 ? left : (n - 1) + ~left] = i;
        parent[right >= 0 ? right : (n - 1) + ~right] = i;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) parent[0] = -1;   // the root (internal node 0, or the only leaf)
}

// Bottom-up boxes: node slots 0..n-2 internal, n-1+s leaf s (sorted order).
// The second child to arrive at a node (atomic counter) merges its two boxes.
// Block b takes the kRefitChunk leaves from s0 = b * kRefitChunk; an inner
// node whose leaf range (rng, from k_karras) lies inside that chunk has
// its index there too (a Karras node's index is an end of its range), so
// its counter and box live in the block's shared memory: the lower levels
// of the climb hand over at shared-memory latency, and only the nodes that
// straddle chunks take the device-wide counter and fences.  The boxes are
// minima and maxima, so the merge order changes no bit of them.
constexpr int kRefitChunk = 256;
// fetch-and-add with release (this thread's earlier writes are visible
// before the add) and acquire (writes released by earlier adds are visible
// after it) at device scope
__device__ __forceinline__ int atomic_add_acq_rel(int* p, int v) {
    int old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
__global__ void __launch_bounds__(kRefitChunk) k_refit(const double* leaf_box, const int* ids, int n, const int* child,
                                                       const int* parent, const int2* rng, double* nbox, int* flags) {
    __shared__ double sbox[2 * kRefitChunk][6];   // [0, C): inner nodes s0.., [C, 2C): leaves s0..
    __shared__ int sflag[kRefitChunk];
    const int s0 = blockIdx.x * kRefitChunk, s = s0 + threadIdx.x;
    sflag[threadIdx.x] = 0;
    __syncthreads();
    if (s >= n) return;
    const int last = min(s0 + kRefitChunk, n) - 1;
    double b[6];
    const double* src = leaf_box + 6 * (size_t)ids[s];
    double* lb = nbox + 6 * ((size_t)(n - 1) + s);
    for (int a = 0; a < 6; ++a) { b[a] = src[a]; lb[a] = b[a]; sbox[kRefitChunk + threadIdx.x][a] = b[a]; }
    if (n == 1) return;
    auto slot = [&](int ch) { return ch >= 0 ? ch - s0 : kRefitChunk + (~ch - s0); };
    bool local = true;
    int from = ~s;   // the child this thread arrives from; its box is b
    int node = parent[(n - 1) + s];
    for (int guard = 0; node >= 0 && guard < 64 + n; ++guard) {
        const int c0 = child[2 * node], c1 = child[2 * node + 1];
        const int sib = c0 == from ? c1 : c0;
        if (local) {
            const int2 r = rng[node];
            local = r.x >= s0 && r.y <= last;
        }
        double o[6];
        if (local) {
            __threadfence_block();
            if (atomicAdd_block(&sflag[node - s0], 1) == 0) return;   // first arrival: the sibling finishes
            __threadfence_block();
            for (int a = 0; a < 6; ++a) o[a] = sbox[slot(sib)][a];
        } else {
            if (atomic_add_acq_rel(&flags[node], 1) == 0) return;
            const double* sb = nbox + 6 * (size_t)(sib >= 0 ? sib : (n - 1) + ~sib);
            for (int a = 0; a < 6; ++a) o[a] = __ldcg(sb + a);
        }
        for (int a = 0; a < 3; ++a) {
            b[a] = dmin(b[a], o[a]);
            b[3 + a] = dmax(b[3 + a], o[3 + a]);
        }
        if (local)
            for (int a = 0; a < 6; ++a) sbox[node - s0][a] = b[a];
        double* bn = nbox + 6 * (size_t)node;
        for (int a = 0; a < 6; ++a) bn[a] = b[a];
        from = node;
        node = parent[node];
    }
}

__device__ __forceinline__ bool boxes_overlap(const double* a, const double* b) {
    return a[0] <= b[3] && b[0] <= a[3] && a[1] <= b[4] && b[1] <= a[4] && a[2] <= b[5] && b[2] <= a[5];
}

// Small scenes: every query against every primitive box, one warp per query
// testing 32 consecutive primitives per trip; a ballot places each trip's
// hits after the previous trip's in primitive order, so each query's hits
// come out sorted.  The same tests and filters as k_traverse.  mode 0
// counts into cnt, mode 1 writes at off.
__global__ void k_sweep_all(PrimGeo pg, int kind, const double* qbox, int nq, const double* leaf, int nprim, int* cnt,
                            const int* off, int* out, long long cap = 0x7fffffffffffffffLL) {
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    const long long w0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long qq = w0; qq < nq; qq += nw) {
        const int q = (int)qq;
        double qb[6];
        for (int a = 0; a < 6; ++a) qb[a] = qbox[6 * q + a];
        const int qbody = kind == 0 ? pg.vbody[q] : pg.ebody[q];
        int c = 0;
        int* dst = out ? out + 2 * (size_t)off[q] : nullptr;
        for (int base = kind == 1 ? q + 1 : 0; base < nprim; base += 32) {
            const int prim = base + lane;
            bool hit = false;
            if (prim < nprim) {
                const int pbody = kind == 0 ? pg.fbody[prim] : pg.ebody[prim];
                hit = pbody != qbody && boxes_overlap(qb, leaf + 6 * (size_t)prim);
            }
            const unsigned m = __ballot_sync(0xffffffffu, hit);
            if (hit && dst) {
                const int at = c + __popc(m & below);
                if (off[q] + (long long)at < cap) { dst[2 * at] = q; dst[2 * at + 1] = prim; }   // writes stop at cap pairs
            }
            c += __popc(m);
        }
        if (!out && lane == 0) cnt[q] = c;
    }
}

// Traversal of one query box against the tree; mode 0 counts, mode 1 writes
// the query's hits into its slice in traversal order (sorted afterwards).
// kind 0: vertex queries vs faces (other body); 1: edge queries vs edges
// (other body, query < prim).  Both children's boxes are loaded and tested
// at their parent (independent loads); an overlapping leaf is taken there,
// one overlapping inner child is entered directly and only the second of
// two is pushed.  A leaf is a hit iff its box and every ancestor's box
// overlap the query box, so the hit set does not depend on the order.
// With qorder (edge queries against the edge tree) thread t takes query
// qorder[t], the tree's t-th leaf, so a warp's queries are neighbours in
// space and walk the same nodes.
constexpr int kTravStack = 96;
// In count mode each query's first kQueryBuf hits also go to its row of
// qbuf (traversal order) and a query with more raises *maxq to its count,
// so that a call whose queries all fit copies its lists from qbuf
// (k_copy_slices) instead of traversing again.
__device__ __forceinline__ void load_node_box(const double* p, double b[6]) {
    const double2* p2 = reinterpret_cast<const double2*>(p);   // 48-byte records, 16-byte aligned
    const double2 u = __ldg(p2), v = __ldg(p2 + 1), w = __ldg(p2 + 2);
    b[0] = u.x; b[1] = u.y; b[2] = v.x; b[3] = v.y; b[4] = w.x; b[5] = w.y;
}
// One traversal job: a query kind against its tree.  k_traverse runs two
// jobs in one launch (blocks [0, nb0) the first, the rest the second), so
// the 41 k vertex queries of a mesh scene do not run alone on a mostly idle
// device beside the edge queries.
struct TravJob {
    int kind;
    const double* qbox; int nq;
    const double* nbox; const int* child; const int* ids; int n;
    int* cnt; const int* off; int* out; int* maxq; int* qbuf; const int* qorder;
};
__device__ __forceinline__ void traverse_job(const PrimGeo& pg, const TravJob& j, int t0, int stride, int* status) {
    const int kind = j.kind, nq = j.nq, n = j.n;
    const double* qbox = j.qbox;
    const double* nbox = j.nbox;
    const int* ids = j.ids;
    const int* off = j.off;
    int* out = j.out;
    int* qbuf = j.qbuf;
    const int* qorder = j.qorder;
    const int2* ch2 = reinterpret_cast<const int2*>(j.child);
    for (int t = t0; t < nq; t += stride) {
        const int q = qorder ? qorder[t] : t;
        double qb[6];
        for (int a = 0; a < 6; ++a) qb[a] = qbox[6 * q + a];
        const int qbody = kind == 0 ? pg.vbody[q] : pg.ebody[q];
        int c = 0;
        int* dst = out ? out + 2 * (size_t)off[q] : nullptr;
        auto leaf_hit = [&](int leaf) {
            const int prim = ids[leaf];
            const int pbody = kind == 0 ? pg.fbody[prim] : pg.ebody[prim];
            if (pbody == qbody || (kind == 1 && !(q < prim))) return;
            if (dst) {
                dst[2 * c] = q;
                dst[2 * c + 1] = prim;
            } else if (qbuf && c < kQueryBuf) {
                qbuf[(size_t)kQueryBuf * q + c] = prim;
            }
            ++c;
        };
        double rb[6];
        load_node_box(nbox, rb);   // slot 0: the root (inner node 0, or the single leaf)
        if (boxes_overlap(qb, rb)) {
            if (n == 1) {
                leaf_hit(0);
            } else {
                int stack[kTravStack];
                int top = 0, node = 0;
                for (;;) {
                    const int2 cc = __ldg(ch2 + node);
                    double bl[6], br[6];
                    load_node_box(nbox + 6 * (size_t)(cc.x >= 0 ? cc.x : (n - 1) + ~cc.x), bl);
                    load_node_box(nbox + 6 * (size_t)(cc.y >= 0 ? cc.y : (n - 1) + ~cc.y), br);
                    const bool ol = boxes_overlap(qb, bl), orr = boxes_overlap(qb, br);
                    if (ol && cc.x < 0) leaf_hit(~cc.x);
                    if (orr && cc.y < 0) leaf_hit(~cc.y);
                    const bool dl = ol && cc.x >= 0, dr = orr && cc.y >= 0;
                    if (dl && dr) {
                        if (top < kTravStack) stack[top++] = cc.y;
                        else atomicExch(status, NXD_CAPACITY);
                        node = cc.x;
                    } else if (dl) {
                        node = cc.x;
                    } else if (dr) {
                        node = cc.y;
                    } else if (top > 0) {
                        node = stack[--top];
                    } else {
                        break;
                    }
                }
            }
        }
        if (!out) {
            j.cnt[q] = c;
            if (c > kQueryBuf) atomicMax(j.maxq, c);
        }
    }
}
__global__ void k_traverse(PrimGeo pg, TravJob j0, TravJob j1, int nb0, int* status) {
    if ((int)blockIdx.x < nb0) traverse_job(pg, j0, blockIdx.x * blockDim.x + threadIdx.x, nb0 * blockDim.x, status);
    else traverse_job(pg, j1, (blockIdx.x - nb0) * blockDim.x + threadIdx.x, (gridDim.x - nb0) * blockDim.x, status);
}

// ---------------------------------------------------------------------------
// Per-pair barrier (PT list then EE list), chained to body DOFs.
// ---------------------------------------------------------------------------
struct IpcPairs {
    const int* pt; int n_pt;
    const int* ee; int n_ee;
};

struct IpcPose {
    const double* wq;      // world vertices at x [nv*3]
    const double* pp;      // body positions at x [N*3]
    const double* x;       // the iterate [6N] (rotation vectors theta), or null: theta = 0
};
__device__ __forceinline__ V3 pose_theta(const IpcPose& ps, int b) {
    return ps.x ? ld3(ps.x + 6 * b + 3) : v3(0, 0, 0);
}

__device__ __forceinline__ void pair_points(const PrimGeo& pg, const IpcPairs& P, const IpcPose& ps, int p, int& kind,
                                            V3* X, int* side, V3* arm, int& bA, int& bB) {
    int vid[4];
    if (p < P.n_pt) {
        kind = ipc::kPairPT;
        const int v = P.pt[2 * p], f = P.pt[2 * p + 1];
        vid[0] = v; vid[1] = pg.fvert[3 * f]; vid[2] = pg.fvert[3 * f + 1]; vid[3] = pg.fvert[3 * f + 2];
        bA = pg.vbody[v]; bB = pg.fbody[f];
        side[0] = 0; side[1] = 1; side[2] = 1; side[3] = 1;
    } else {
        kind = ipc::kPairEE;
        const int q = p - P.n_pt;
        const int e0 = P.ee[2 * q], e1 = P.ee[2 * q + 1];
        vid[0] = pg.evert[2 * e0]; vid[1] = pg.evert[2 * e0 + 1]; vid[2] = pg.evert[2 * e1]; vid[3] = pg.evert[2 * e1 + 1];
        bA = pg.ebody[e0]; bB = pg.ebody[e1];
        side[0] = 0; side[1] = 0; side[2] = 1; side[3] = 1;
    }
    for (int k = 0; k < 4; ++k) {
        X[k] = ld3(ps.wq + 3 * vid[k]);
        arm[k] = X[k] - ld3(ps.pp + 3 * (side[k] ? bB : bA));
    }
}

struct IpcEvalOut {
    double* e;         // [n] pair energy
    double* grad;      // [n*12] chained gradient (A 0..5, B 6..11)
    double* lam;       // [n*5]
    double* z;         // [n*5*12]
    int* nterm;        // [n]
    int* body;         // [n*2]
    int* active;       // [n] 1 when d^2 < dhat^2
    int* type;         // [n] distance type
};

__global__ void k_ipc_pair_eval(PrimGeo pg, IpcPairs P, IpcPose ps, double dhat, double kappa, IpcEvalOut o) {
    const int n = P.n_pt + P.n_ee;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        int kind, side[4], bA, bB;
        V3 X[4], arm[4];
        pair_points(pg, P, ps, p, kind, X, side, arm, bA, bB);
        const ipc::DistForm f = ipc::classify(kind, X);
        const ipc::PairEval ev = ipc::pair_barrier(f, X, dhat, kappa);
        o.e[p] = ev.e;
        o.body[2 * p] = bA; o.body[2 * p + 1] = bB;
        o.type[p] = f.type;
        o.active[p] = ev.d2 < dhat * dhat ? 1 : 0;
        const V3 thA = pose_theta(ps, bA), thB = pose_theta(ps, bB);
        ipc::chain12_exact(ev.grad, side, arm, thA, thB, o.grad + 12 * (size_t)p);
        o.nterm[p] = ev.n_terms;
        for (int k = 0; k < ev.n_terms; ++k) {
            o.lam[5 * (size_t)p + k] = ev.lam[k];
            ipc::chain12_exact(ev.y[k], side, arm, thA, thB, o.z + 60 * (size_t)p + 12 * k);
        }
    }
}

// ---------------------------------------------------------------------------
// Lagged friction (ipc::friction_pair) over a frozen set of pairs: built
// from the active barrier pairs at the lag state (k_fric_lag), evaluated at
// every iterate and trial point (k_fric_eval / k_fric_energy) against the
// step-start world vertices x0.
// ---------------------------------------------------------------------------
struct IpcFric {
    int n;
    int* vid;          // [4n] the pair's four vertices
    int* body;         // [2n] bodies A, B
    int* kind;         // [n]  ipc::kPairPT / kPairEE (fixes the sides)
    double* w;         // [4n] closest-point weights
    double* nrm;       // [3n] unit normal
    double* lam;       // [n]  normal force
    const double* x0;  // step-start world vertices [nv*3]
};

__device__ __forceinline__ void pair_vids(const PrimGeo& pg, const IpcPairs& P, int p, int* vid, int& kind, int& bA, int& bB) {
    if (p < P.n_pt) {
        kind = ipc::kPairPT;
        const int v = P.pt[2 * p], f = P.pt[2 * p + 1];
        vid[0] = v; vid[1] = pg.fvert[3 * f]; vid[2] = pg.fvert[3 * f + 1]; vid[3] = pg.fvert[3 * f + 2];
        bA = pg.vbody[v]; bB = pg.fbody[f];
    } else {
        kind = ipc::kPairEE;
        const int q = p - P.n_pt;
        const int e0 = P.ee[2 * q], e1 = P.ee[2 * q + 1];
        vid[0] = pg.evert[2 * e0]; vid[1] = pg.evert[2 * e0 + 1]; vid[2] = pg.evert[2 * e1]; vid[3] = pg.evert[2 * e1 + 1];
        bA = pg.ebody[e0]; bB = pg.ebody[e1];
    }
}
__device__ __forceinline__ void fric_sides(int kind, int* side) {
    side[0] = 0; side[1] = kind == ipc::kPairPT ? 1 : 0; side[2] = 1; side[3] = 1;
}

// The friction set from the active list (pair order) at the lag state.
__global__ void k_fric_lag(PrimGeo pg, IpcPairs P, IpcPose ps, const int* alist, int na, double dhat, double kappa, IpcFric F) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < na; a += gridDim.x * blockDim.x) {
        const int p = alist[a];
        int vid[4], kind, bA, bB;
        pair_vids(pg, P, p, vid, kind, bA, bB);
        V3 X[4];
        for (int k = 0; k < 4; ++k) X[k] = ld3(ps.wq + 3 * vid[k]);
        const ipc::DistForm f = ipc::classify(kind, X);
        ipc::FricLag L;
        ipc::friction_lag(f, X, dhat, kappa, L);
        for (int k = 0; k < 4; ++k) { F.vid[4 * a + k] = vid[k]; F.w[4 * a + k] = L.w[k]; }
        F.body[2 * a] = bA; F.body[2 * a + 1] = bB;
        F.kind[a] = kind;
        F.nrm[3 * a] = L.n.x; F.nrm[3 * a + 1] = L.n.y; F.nrm[3 * a + 2] = L.n.z;
        F.lam[a] = L.lam;
    }
}

__device__ __forceinline__ ipc::FricEval fric_at(const IpcFric& F, const IpcPose& ps, int f, double mu, double eps, int* side,
                                                 V3* arm, int& bA, int& bB) {
    ipc::FricLag L;
    V3 X[4], X0[4];
    bA = F.body[2 * f]; bB = F.body[2 * f + 1];
    fric_sides(F.kind[f], side);
    for (int k = 0; k < 4; ++k) {
        const int v = F.vid[4 * f + k];
        X[k] = ld3(ps.wq + 3 * v);
        X0[k] = ld3(F.x0 + 3 * v);
        arm[k] = X[k] - ld3(ps.pp + 3 * (side[k] ? bB : bA));
        L.w[k] = F.w[4 * f + k];
    }
    L.n = ld3(F.nrm + 3 * f);
    L.lam = F.lam[f];
    return ipc::friction_pair(L, X, X0, mu, eps);
}

// Friction pair f into slot base + f of the pair arrays (gradient, two
// Hessian terms, bodies) and its energy into ef[f].
__global__ void k_fric_eval(IpcFric F, IpcPose ps, double mu, double eps, int base, double* ef, IpcEvalOut o) {
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < F.n; f += gridDim.x * blockDim.x) {
        int side[4], bA, bB;
        V3 arm[4];
        const ipc::FricEval ev = fric_at(F, ps, f, mu, eps, side, arm, bA, bB);
        const size_t p = (size_t)base + f;
        ef[f] = ev.e;
        o.body[2 * p] = bA; o.body[2 * p + 1] = bB;
        const V3 thA = pose_theta(ps, bA), thB = pose_theta(ps, bB);
        ipc::chain12_exact(ev.grad, side, arm, thA, thB, o.grad + 12 * p);
        o.nterm[p] = 2;
        for (int k = 0; k < 2; ++k) {
            o.lam[5 * p + k] = ev.lam[k];
            ipc::chain12_exact(ev.y[k], side, arm, thA, thB, o.z + 60 * p + 12 * k);
        }
    }
}
__global__ void k_fric_energy(IpcFric F, IpcPose ps, double mu, double eps, double* ef) {
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < F.n; f += gridDim.x * blockDim.x) {
        int side[4], bA, bB;
        V3 arm[4];
        ef[f] = fric_at(F, ps, f, mu, eps, side, arm, bA, bB).e;
    }
}
// list[at + i] = base + i, i < n (the friction pairs after the active barrier pairs)
__global__ void k_iota(int* list, const int* at, int base, int n) {
    const int o = *at;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) list[o + i] = base + i;
}

// Step adjoint, per candidate pair at the converged iterate: the exact
// derivative of the pair's share of the step gradient G (point forces g_k,
// torques J_r(theta) sum a_k x g_k) with respect to the two bodies' DOFs
// (kp, 12 x 12: rows and columns A 0..5, B 6..11) and to left rotations phi
// of their step-start orientations (kf, 12 x 6: columns phi_A, phi_B):
//   kp = E^T H E + Q,  kf = E^T H F + Q_phi,
// H the unprojected point Hessian (ipc::pair_barrier_exact), E_k = [I,
// -[a_k]x J_l(theta)] and F_k = -[a_k]x Exp(theta) the points' derivatives,
// Q = J_r (sum_k [g_k]x [a_k]x) J_l + d(J_r tau)/dtheta and Q_phi =
// J_r (sum_k [g_k]x [a_k]x) Exp(theta) on each body's own rotation block.
// Unscaled (the step scales the barrier by s); inactive pairs flagged 0.
// The pair's share of dG/dx (KP, 12 x 12) and dG/dphi (KF, 12 x 6) for
// point forces g12 with point Jacobian H (row 3k+i, column 3l+j), points of
// bodies side[k] at arms arm[k], body rotations th; E (12 x 12) receives the
// point-velocity map [I, -[a]x J_l(theta)].
__device__ void pair_adjoint_blocks(const double* g12, const double* H, const int* side, const V3* arm, const V3* th,
                                    double* KP, double* KF, double* E) {
    double R[2][9], Jl[2][9];
    for (int sd = 0; sd < 2; ++sd) ipc::rot_exp_mats(th[sd], R[sd], Jl[sd]);
    double F[72];
    for (int e = 0; e < 144; ++e) E[e] = 0.0;
    for (int e = 0; e < 72; ++e) F[e] = 0.0;
    for (int k = 0; k < 4; ++k) {
        const int sg = side[k];
        double A[9], D[9], Fk[9];
        ipc::m3_skew(arm[k], A);
        ipc::m3_mul(A, Jl[sg], D);
        ipc::m3_mul(A, R[sg], Fk);
        for (int i = 0; i < 3; ++i) {
            E[12 * (3 * k + i) + 6 * sg + i] = 1.0;
            for (int j = 0; j < 3; ++j) {
                E[12 * (3 * k + i) + 6 * sg + 3 + j] = -D[3 * i + j];
                F[6 * (3 * k + i) + 3 * sg + j] = -Fk[3 * i + j];
            }
        }
    }
    for (int r = 0; r < 12; ++r) {
        double he[12], hf[6];
        for (int c = 0; c < 12; ++c) he[c] = 0.0;
        for (int c = 0; c < 6; ++c) hf[c] = 0.0;
        // rows of E^T H: sum_i E[i][r] H[i][.]
        for (int i = 0; i < 12; ++i) {
            const double eir = E[12 * i + r];
            if (eir == 0.0) continue;
            for (int j = 0; j < 12; ++j) {
                const double t = eir * H[12 * i + j];
                for (int c = 0; c < 12; ++c) he[c] += t * E[12 * j + c];
                for (int c = 0; c < 6; ++c) hf[c] += t * F[6 * j + c];
            }
        }
        for (int c = 0; c < 12; ++c) KP[12 * r + c] = he[c];
        for (int c = 0; c < 6; ++c) KF[6 * r + c] = hf[c];
    }
    for (int sg = 0; sg < 2; ++sg) {
        double GA[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        V3 tau = v3(0, 0, 0);
        for (int k = 0; k < 4; ++k) {
            if (side[k] != sg) continue;
            const V3 gk = v3(g12[3 * k], g12[3 * k + 1], g12[3 * k + 2]);
            double SG[9], SA[9], P9[9];
            ipc::m3_skew(gk, SG);
            ipc::m3_skew(arm[k], SA);
            ipc::m3_mul(SG, SA, P9);
            for (int e = 0; e < 9; ++e) GA[e] += P9[e];
            tau = tau + cross(arm[k], gk);
        }
        double Jr[9], T1[9], Q[9], QF[9], M[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) Jr[3 * i + j] = Jl[sg][3 * j + i];
        ipc::m3_mul(Jr, GA, T1);
        ipc::m3_mul(T1, Jl[sg], Q);
        ipc::m3_mul(T1, R[sg], QF);
        ipc::jr_torque_derivative(th[sg], tau, M);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                KP[12 * (6 * sg + 3 + i) + 6 * sg + 3 + j] += Q[3 * i + j] + M[3 * i + j];
                KF[6 * (6 * sg + 3 + i) + 3 * sg + j] += QF[3 * i + j];
            }
    }
}

__global__ void k_ipc_pair_adjoint(PrimGeo pg, IpcPairs P, IpcPose ps, double dhat, double kappa, double* kp, double* kf,
                                   int* body, int* active) {
    const int n = P.n_pt + P.n_ee;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        int kind, side[4], bA, bB;
        V3 X[4], arm[4];
        pair_points(pg, P, ps, p, kind, X, side, arm, bA, bB);
        const ipc::DistForm f = ipc::classify(kind, X);
        double g12[12], H[144];
        const double d2 = ipc::pair_barrier_exact(f, X, dhat, kappa, g12, H);
        body[2 * p] = bA; body[2 * p + 1] = bB;
        const bool act = d2 < dhat * dhat && d2 > 0.0;
        active[p] = act ? 1 : 0;
        if (!act) continue;
        const V3 th[2] = {pose_theta(ps, bA), pose_theta(ps, bB)};
        double E[144];
        pair_adjoint_blocks(g12, H, side, arm, th, kp + 144 * (size_t)p, kf + 72 * (size_t)p, E);
    }
}

// Step adjoint of the lagged friction, per frozen pair at the converged
// iterate: kp / kf as for the barrier (ipc::friction_derivs' point forces
// and H), ks (12 x 12, columns p_A, phi_A, p_B, phi_B) = E^T Hs S with S the
// step-start points' derivatives ([I, -[a_s]x] per point, a_s the
// step-start arm: the lag state moves with the start positions and, on the
// left, orientations) and gm (12) = E^T F / mu, the derivative in mu.
// Unscaled; the frozen set and its step-start points as the step built them.
__global__ void k_fric_pair_adjoint(IpcFric Fz, IpcPose ps, const double* pos0, double dhat, double kappa, double mu,
                                    double eps, double* kp, double* kf, double* ks, double* gm, int* body) {
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < Fz.n; f += gridDim.x * blockDim.x) {
        int side[4];
        const int bA = Fz.body[2 * f], bB = Fz.body[2 * f + 1];
        const int kind = Fz.kind[f];
        fric_sides(kind, side);
        V3 X[4], Xs[4], arm[4], arm_s[4];
        const int b[2] = {bA, bB};
        for (int k = 0; k < 4; ++k) {
            const int v = Fz.vid[4 * f + k];
            X[k] = ld3(ps.wq + 3 * v);
            Xs[k] = ld3(Fz.x0 + 3 * v);
            arm[k] = X[k] - ld3(ps.pp + 3 * b[side[k]]);
            arm_s[k] = Xs[k] - ld3(pos0 + 3 * b[side[k]]);
        }
        const ipc::DistForm fs = ipc::classify(kind, Xs);
        double g12[12], H[144], Hs[144];
        ipc::friction_derivs(fs, X, Xs, dhat, kappa, mu, eps, g12, H, Hs);
        body[2 * f] = bA; body[2 * f + 1] = bB;
        const V3 th[2] = {pose_theta(ps, bA), pose_theta(ps, bB)};
        double E[144];
        pair_adjoint_blocks(g12, H, side, arm, th, kp + 144 * (size_t)f, kf + 72 * (size_t)f, E);
        // S: step-start points from (p_A, phi_A, p_B, phi_B)
        double S[144];
        for (int e = 0; e < 144; ++e) S[e] = 0.0;
        for (int k = 0; k < 4; ++k) {
            const int sg = side[k];
            double A[9];
            ipc::m3_skew(arm_s[k], A);
            for (int i = 0; i < 3; ++i) {
                S[12 * (3 * k + i) + 6 * sg + i] = 1.0;
                for (int j = 0; j < 3; ++j) S[12 * (3 * k + i) + 6 * sg + 3 + j] = -A[3 * i + j];
            }
        }
        double* KS = ks + 144 * (size_t)f;
        for (int r = 0; r < 12; ++r) {
            double hs[12];
            for (int c = 0; c < 12; ++c) hs[c] = 0.0;
            for (int i = 0; i < 12; ++i) {
                const double eir = E[12 * i + r];
                if (eir == 0.0) continue;
                for (int j = 0; j < 12; ++j) {
                    const double t = eir * Hs[12 * i + j];
                    for (int c = 0; c < 12; ++c) hs[c] += t * S[12 * j + c];
                }
            }
            for (int c = 0; c < 12; ++c) KS[12 * r + c] = hs[c];
            double gr = 0.0;
            for (int i = 0; i < 12; ++i) gr += E[12 * i + r] * g12[i];
            gm[12 * (size_t)f + r] = gr / mu;
        }
    }
}

// Energy only (line-search trial points): the same classification and
// barrier value as k_ipc_pair_eval's e, without the PSD projection.
__global__ void k_ipc_pair_energy(PrimGeo pg, IpcPairs P, IpcPose ps, double dhat, double kappa, double* e) {
    const int n = P.n_pt + P.n_ee;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        int kind, side[4], bA, bB;
        V3 X[4], arm[4];
        pair_points(pg, P, ps, p, kind, X, side, arm, bA, bB);
        const ipc::DistForm f = ipc::classify(kind, X);
        const V3 r = ipc::form_r(f, X);
        e[p] = ipc::barrier_s(dot(r, r), dhat * dhat, kappa);
    }
}

// k_ipc_pair_energy with the pair counts read on the device (tot[0] point-
// triangle, tot[1] edge-edge); lists over their capacities (cap_pt, cap_ee
// pairs) are left alone, the caller sees the totals and evaluates again.
__global__ void k_ipc_pair_energy_dev(PrimGeo pg, const int* pt, const int* ee, const int* tot, int cap_pt, int cap_ee,
                                      IpcPose ps, double dhat, double kappa, double* e, const int* guard = nullptr) {
    const int npt = tot[0], nee = tot[1];
    if (npt > cap_pt || nee > cap_ee || (guard && (guard[0] | guard[1]))) return;
    const IpcPairs P{pt, npt, ee, nee};
    const int n = npt + nee;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        int kind, side[4], bA, bB;
        V3 X[4], arm[4];
        pair_points(pg, P, ps, p, kind, X, side, arm, bA, bB);
        const ipc::DistForm f = ipc::classify(kind, X);
        const V3 r = ipc::form_r(f, X);
        e[p] = ipc::barrier_s(dot(r, r), dhat * dhat, kappa);
    }
}

// Contributions of the active pairs: gradient (body, pair, side) and
// Hessian blocks (row body, col body, pair, block) with their segment keys.
__global__ void k_ipc_contrib(const int* active_list, int na, const int* body, int N, unsigned long long* gkey, int* gval,
                              unsigned long long* hkey, int* hval) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < na; a += gridDim.x * blockDim.x) {
        const int p = active_list[a];
        const int b[2] = {body[2 * p], body[2 * p + 1]};
        for (int s = 0; s < 2; ++s) {
            gkey[2 * a + s] = (unsigned long long)b[s];
            gval[2 * a + s] = 2 * p + s;
        }
        for (int r = 0; r < 2; ++r)
            for (int c = 0; c < 2; ++c) {
                hkey[4 * a + 2 * r + c] = (unsigned long long)b[r] * (unsigned long long)N + (unsigned long long)b[c];
                hval[4 * a + 2 * r + c] = 4 * p + 2 * r + c;
            }
    }
}

// Segment starts of sorted keys: flag[i] = key changes at i.
__global__ void k_seg_flags(const unsigned long long* key, int n, int* flag) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        flag[i] = (i == 0 || key[i] != key[i - 1]) ? 1 : 0;
}
__global__ void k_seg_starts(const int* flag, const int* pos, int n, int* start, int* nseg) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (flag[i]) start[pos[i]] = i;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const int m = n > 0 ? pos[n - 1] + flag[n - 1] : 0;
        *nseg = m;
        start[m] = n;
    }
}

// Segment sums of the barrier's gradient and Hessian blocks, in one fixed
// order on the device and in the oracle: a segment of m <= kSegSerial
// contributions (pair order) is summed left to right from 0; a longer one
// as 32 partial sums, partial l taking the contributions i = l (mod 32) left
// to right, then halved pairwise (a_l += a_{l+16}, ..., a_0 += a_1).  Light
// segments take a thread each; heavy ones (a body touching many pairs, such
// as a static container) a warp each, so their cost is m / 32 dependent
// adds instead of m.
constexpr int kSegSerial = 32;

__device__ __forceinline__ double ipc_grad_term(const int* gval, const double* pgrad, int i, int dof) {
    const int v = gval[i];
    return pgrad[12 * (size_t)(v >> 1) + 6 * (v & 1) + dof];
}
__device__ __forceinline__ double ipc_hess_term(const int* hval, const double* lam, const double* z, const int* nterm, int s, int i,
                                                int j) {
    const int v = hval[s];
    const int p = v >> 2, r = (v >> 1) & 1, c = v & 1;
    double blk = 0.0;
    for (int k = 0; k < nterm[p]; ++k) {
        const double* zk = z + 60 * (size_t)p + 12 * k;
        blk += (lam[5 * (size_t)p + k] * zk[6 * r + i]) * zk[6 * c + j];
    }
    return blk;
}
// lanes' partials halved pairwise into lane 0
__device__ __forceinline__ double warp_halve_sum(double a) {
    const int lane = threadIdx.x & 31;
    for (int off = 16; off >= 1; off >>= 1) {
        const double o = __shfl_down_sync(0xffffffffu, a, off);
        if (lane < off) a += o;
    }
    return a;
}

// Gradient, light segments: thread per (segment, dof).
__global__ void k_ipc_grad(const unsigned long long* gkey, const int* gval, const int* start, const int* nseg, const double* pgrad,
                           double* grad) {
    const int ns = *nseg;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 6 * ns; t += gridDim.x * blockDim.x) {
        const int sgm = t / 6, dof = t % 6;
        if (start[sgm + 1] - start[sgm] > kSegSerial) continue;
        double acc = 0.0;
        for (int i = start[sgm]; i < start[sgm + 1]; ++i) acc += ipc_grad_term(gval, pgrad, i, dof);
        grad[6 * gkey[start[sgm]] + dof] = acc;
    }
}
// Gradient, heavy segments: warp per (segment, dof), warps striding over all.
__global__ void k_ipc_grad_heavy(const unsigned long long* gkey, const int* gval, const int* start, const int* nseg,
                                 const double* pgrad, double* grad) {
    const int ns = *nseg, lane = threadIdx.x & 31;
    const long long w0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long t = w0; t < 6LL * ns; t += nw) {
        const int sgm = (int)(t / 6), dof = (int)(t % 6);
        const int a = start[sgm], b = start[sgm + 1];
        if (b - a <= kSegSerial) continue;
        double acc = 0.0;
        for (int i = a + lane; i < b; i += 32) acc += ipc_grad_term(gval, pgrad, i, dof);
        acc = warp_halve_sum(acc);
        if (lane == 0) grad[6 * gkey[a] + dof] = acc;
    }
}

// Hessian blocks: block (r, c) of pair p is sum_k (lam_k z_k[r-side i])
// z_k[c-side j]; each block entry is its segment's sum in the order above.
// Writes BSR col_idx / vals in sorted (row, col) order.  Light segments:
// thread per (segment, entry).
__global__ void k_ipc_hess(const unsigned long long* hkey, const int* hval, const int* start, const int* nseg, int N,
                           const double* lam, const double* z, const int* nterm, int* col_idx, double* vals, long long cap) {
    const int ns = *nseg;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 36 * ns; t += gridDim.x * blockDim.x) {
        const int sgm = t / 36, e = t % 36, i = e / 6, j = e % 6;
        if (sgm >= cap) continue;
        if (e == 0) col_idx[sgm] = (int)(hkey[start[sgm]] % (unsigned long long)N);
        if (start[sgm + 1] - start[sgm] > kSegSerial) continue;
        double acc = 0.0;
        for (int s = start[sgm]; s < start[sgm + 1]; ++s) acc += ipc_hess_term(hval, lam, z, nterm, s, i, j);
        vals[36 * (size_t)sgm + e] = acc;
    }
}
// Hessian blocks, heavy segments: warp per (segment, entry).
__global__ void k_ipc_hess_heavy(const int* hval, const int* start, const int* nseg, const double* lam, const double* z,
                                 const int* nterm, double* vals, long long cap) {
    const int ns = *nseg, lane = threadIdx.x & 31;
    const long long w0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long t = w0; t < 36LL * ns; t += nw) {
        const int sgm = (int)(t / 36), e = (int)(t % 36), i = e / 6, j = e % 6;
        if (sgm >= cap) continue;
        const int a = start[sgm], b = start[sgm + 1];
        if (b - a <= kSegSerial) continue;
        double acc = 0.0;
        for (int s = a + lane; s < b; s += 32) acc += ipc_hess_term(hval, lam, z, nterm, s, i, j);
        acc = warp_halve_sum(acc);
        if (lane == 0) vals[36 * (size_t)sgm + e] = acc;
    }
}

__global__ void k_ipc_rowptr(const unsigned long long* hkey, const int* start, const int* nseg, int N, int* row_ptr) {
    const int ns = *nseg;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r <= N; r += gridDim.x * blockDim.x) {
        // first segment whose row >= r (binary search over sorted segment keys)
        int lo = 0, hi = ns;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if ((long long)(hkey[start[mid]] / (unsigned long long)N) < r) lo = mid + 1;
            else hi = mid;
        }
        row_ptr[r] = lo;
    }
}

// ---------------------------------------------------------------------------
// Additive CCD over the candidate pairs (swept boxes): per pair the time of
// impact along its points' motion (ipc::accd_toi_motion; the step uses the
// rigid arcs, ipc::ArcMotion), then the minimum (one block).  A thread per
// pair evaluates its Lipschitz bound and start distance and settles the
// pairs whose first safe advance already reaches t_max (most candidates of
// a step); the pairs left are appended to a list (k_ipc_accd), and a warp
// per listed pair then samples kAccdLookahead points a round in its lanes
// (k_ipc_accd_rounds).  The arithmetic per pair is accd_toi_motion's, so
// the bound is the same, whichever warp takes which pair.
// ---------------------------------------------------------------------------
static_assert(ipc::kAccdLookahead == 32, "one sample per lane");
template <typename M>
__device__ double accd_toi_warp(const M& m, double lp, double d0, double t_max, double eta, int max_iter) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const double g = eta * d0;
    double t = 0.0, d = d0;
    for (int it = 0; it < max_iter; ++it) {
        const double dl = 0.9 * (d - g) / lp;
        if (t + dl >= t_max) return t_max;
        if (!(dl > 1e-12 * t_max)) return t;
        const double thr = g + 0.9 * (d - g);
        const double tj = t + (double)(lane + 1) * dl;
        const bool past = tj >= t_max;
        const double dj = past ? 0.0 : m.distance(tj);
        // the round ends at the first sample past t_max or below thr
        const unsigned stop = __ballot_sync(full, past || !(dj >= thr));
        const int J = stop ? __ffs(stop) - 1 : 31;
        if ((stop >> J) & 1u) {
            if (__shfl_sync(full, past ? 1 : 0, J)) return t_max;
        }
        t = __shfl_sync(full, tj, J);
        d = __shfl_sync(full, dj, J);
    }
    return t;
}

// Time of impact of each candidate pair along the rigid arcs x + t dx
// (ipc::ArcMotion: body-local vertices vloc, step-start orientations q0).
__device__ __forceinline__ void arc_motion_of(const PrimGeo& pg, const IpcPairs& P, int p, const double* vloc,
                                              const double* x, const double* dx, const double* q0, ipc::ArcMotion& m) {
    int vid[4], kind, bA, bB;
    pair_vids(pg, P, p, vid, kind, bA, bB);
    m.kind = kind;
    fric_sides(kind, m.side);
    const int b[2] = {bA, bB};
    for (int sd = 0; sd < 2; ++sd) {
        m.b[sd].p = ld3(x + 6 * b[sd]);
        m.b[sd].th = ld3(x + 6 * b[sd] + 3);
        m.b[sd].dp = ld3(dx + 6 * b[sd]);
        m.b[sd].dth = ld3(dx + 6 * b[sd] + 3);
        m.b[sd].q0 = ldq(q0 + 4 * b[sd]);
    }
    for (int k = 0; k < 4; ++k) m.v[k] = ld3(vloc + 3 * vid[k]);
}
__global__ void k_ipc_accd(PrimGeo pg, IpcPairs P, const double* vloc, const double* x, const double* dx, const double* q0,
                           double eta, int max_iter, double* toi, int* list, double2* lpd0, int* nlist) {
    const unsigned full = 0xffffffffu;
    const double t_max = 1.0;
    const int n = P.n_pt + P.n_ee;
    const int lane = threadIdx.x & 31;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long base = (long long)blockIdx.x * blockDim.x + threadIdx.x - lane; base < n; base += stride) {
        const int p = (int)base + lane;
        double lp = 0.0, d0 = 0.0;
        bool need = false;
        if (p < n) {
            ipc::ArcMotion m;
            arc_motion_of(pg, P, p, vloc, x, dx, q0, m);
            lp = m.lipschitz();
            d0 = m.distance(0.0);
            // accd_toi_motion's exits before its first round of samples
            double res = 0.0;
            if (!(lp > 0.0)) {
                res = t_max;
            } else if (d0 > 0.0 && max_iter > 0) {
                const double dl = 0.9 * (d0 - eta * d0) / lp;
                if (0.0 + dl >= t_max) res = t_max;
                else need = dl > 1e-12 * t_max;
            }
            if (!need) toi[p] = res;
        }
        const unsigned todo = __ballot_sync(full, need);
        if (!todo) continue;
        int at = 0;
        if (lane == 0) at = atomicAdd(nlist, __popc(todo));
        at = __shfl_sync(full, at, 0) + __popc(todo & ((1u << lane) - 1u));
        if (need) {
            list[at] = p;
            lpd0[at] = make_double2(lp, d0);
        }
    }
}
// One warp per listed pair: accd_toi_motion's rounds from its start.
__global__ void k_ipc_accd_rounds(PrimGeo pg, IpcPairs P, const double* vloc, const double* x, const double* dx,
                                  const double* q0, double eta, int max_iter, const int* list, const double2* lpd0,
                                  const int* nlist, double* toi) {
    const int m_ = *nlist;
    const long long w0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long k = w0; k < m_; k += nw) {
        const int p = list[k];
        const double2 ld = lpd0[k];
        ipc::ArcMotion m;
        arc_motion_of(pg, P, p, vloc, x, dx, q0, m);
        const double tp = accd_toi_warp(m, ld.x, ld.y, 1.0, eta, max_iter);
        if ((threadIdx.x & 31) == 0) toi[p] = tp;
    }
}

__global__ void k_min_reduce(const double* v, int n, double init, double* out) {
    __shared__ double sm[32];
    double m = init;
    for (int i = threadIdx.x; i < n; i += blockDim.x) m = dmin(m, v[i]);
    for (int o = 16; o > 0; o >>= 1) m = dmin(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = init;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) r = dmin(r, sm[k]);
        *out = r;
    }
}

// max |v_i| over n doubles, one block; a NaN entry makes the result NaN.
__global__ void k_absmax(const double* v, int n, double* out) {
    __shared__ double sm[32];
    double m = 0.0;
    auto fold = [](double a, double b) { return a != a ? a : ((b != b || b > a) ? b : a); };
    for (int i = threadIdx.x; i < n; i += blockDim.x) m = fold(m, fabs(v[i]));
    for (int o = 16; o > 0; o >>= 1) m = fold(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) r = fold(r, sm[k]);
        *out = r;
    }
}

// k_tree_sum of the n = tot[0] + tot[1] pair energies (nothing when the
// lists overflowed their capacities, see k_ipc_pair_energy_dev).
__global__ void __launch_bounds__(1024) k_tree_sum_pairs(const double* v, const int* tot, int cap_pt, int cap_ee, double* out) {
    __shared__ double sh[2 * kRedMaxQ * 32];
    if (tot[0] > cap_pt || tot[1] > cap_ee) return;
    BlockRed R;
    R.sh = sh;
    R.parity = 0;
    const double s = R.sum(tot[0] + tot[1], [&](int e) { return v[e]; });
    if (threadIdx.x == 0) *out = s;
}

// Fixed-tree sum of n doubles (the padded pairwise tree), one block.
__global__ void __launch_bounds__(1024) k_tree_sum(const double* v, int n, double* out) {
    __shared__ double sh[2 * kRedMaxQ * 32];
    BlockRed R;
    R.sh = sh;
    R.parity = 0;
    const double s = R.sum(n, [&](int e) { return v[e]; });
    if (threadIdx.x == 0) *out = s;
}

}  // namespace nx
