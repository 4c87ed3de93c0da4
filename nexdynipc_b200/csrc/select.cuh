// select.cuh — warp-parallel, permutation-exact emulation of
//   std::nth_element(first, first + k, last, comp);  std::sort(first, first + k, comp);
// as implemented by GCC 13's libstdc++ (introselect / introsort with
// median-of-three Hoare partitioning, insertion-sort finish and heap
// fallbacks), which select_top_k_indices calls
// (nexdynipc/src/Physics/Contact/ContactAssembler.cpp:67-88).
//
// Ties are frequent there (every vertex inside the other body's box scores 0),
// so the chosen subset depends on the library's data movement; reproducing it
// is what makes the candidate sets identical to the CPU path.
//
// Data-parallel form of one Hoare partition of [first+1, last) around the
// pivot at `first` (libstdc++ __unguarded_partition):
//   G = ascending positions p in [first+1, last) with !(key[p] < pivot)
//   L = descending positions p in [first, last)   with !(pivot < key[p])
// The sequential scan swaps G[t] <-> L[t] for t = 0..m-1, where m is the
// number of t with G[t] < L[t] (the condition is monotone in t), and returns
// min(G[m], L[m-1]) (missing entries read as +inf).  Proof sketch: untouched
// positions between the two scan pointers are original; each pointer is
// stopped at the latest by the element the previous swap placed behind the
// other pointer, so the t-th stops are exactly G[t] and L[t] until they cross.
//
// The final insertion sort of std::sort is a stable insertion sort of the
// arrangement left by the partitioning (each block is bounded by its
// neighbours), so it is computed here as a stable rank sort.
#pragma once

#include <climits>

namespace nx {

struct SelView {
    int* idx;           // positions -> element id
    const double* key;  // element id -> key
    int* G;             // scratch, capacity n
    int* L;             // scratch, capacity n + 1
};

__device__ __forceinline__ bool sel_less(const SelView& v, int a, int b) { return v.key[a] < v.key[b]; }
__device__ __forceinline__ int lg_floor(int n) { return 31 - __clz(n); }

// ---- serial pieces (lane 0) ------------------------------------------------
__device__ void sel_move_median_to_first(const SelView& v, int result, int a, int b, int c) {
    int* I = v.idx;
    int sw;
    if (sel_less(v, I[a], I[b])) {
        if (sel_less(v, I[b], I[c])) sw = b;
        else if (sel_less(v, I[a], I[c])) sw = c;
        else sw = a;
    } else if (sel_less(v, I[a], I[c])) sw = a;
    else if (sel_less(v, I[b], I[c])) sw = c;
    else sw = b;
    const int t = I[result]; I[result] = I[sw]; I[sw] = t;
}
__device__ void sel_insertion_sort(const SelView& v, int first, int last) {
    int* I = v.idx;
    if (first == last) return;
    for (int i = first + 1; i < last; ++i) {
        const int val = I[i];
        if (sel_less(v, val, I[first])) {
            for (int j = i; j > first; --j) I[j] = I[j - 1];
            I[first] = val;
        } else {
            int j = i;
            while (sel_less(v, val, I[j - 1])) { I[j] = I[j - 1]; --j; }
            I[j] = val;
        }
    }
}
__device__ void sel_adjust_heap(const SelView& v, int first, int hole, int len, int value) {
    int* I = v.idx;
    const int top = hole;
    int second = hole;
    while (second < (len - 1) / 2) {
        second = 2 * (second + 1);
        if (sel_less(v, I[first + second], I[first + second - 1])) second--;
        I[first + hole] = I[first + second];
        hole = second;
    }
    if ((len & 1) == 0 && second == (len - 2) / 2) {
        second = 2 * (second + 1);
        I[first + hole] = I[first + second - 1];
        hole = second - 1;
    }
    int parent = (hole - 1) / 2;
    while (hole > top && sel_less(v, I[first + parent], value)) {
        I[first + hole] = I[first + parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    I[first + hole] = value;
}
__device__ void sel_make_heap(const SelView& v, int first, int last) {
    const int len = last - first;
    if (len < 2) return;
    int parent = (len - 2) / 2;
    while (true) {
        sel_adjust_heap(v, first, parent, len, v.idx[first + parent]);
        if (parent == 0) return;
        parent--;
    }
}
__device__ void sel_pop_heap(const SelView& v, int first, int last, int result) {
    const int value = v.idx[result];
    v.idx[result] = v.idx[first];
    sel_adjust_heap(v, first, 0, last - first, value);
}
__device__ void sel_heap_select(const SelView& v, int first, int middle, int last) {
    sel_make_heap(v, first, middle);
    for (int i = middle; i < last; ++i)
        if (sel_less(v, v.idx[i], v.idx[first])) sel_pop_heap(v, first, middle, i);
}
__device__ void sel_sort_heap(const SelView& v, int first, int last) {
    while (last - first > 1) {
        --last;
        sel_pop_heap(v, first, last, last);
    }
}

// ---- warp-parallel partition ------------------------------------------------
// All 32 lanes call; the pivot is already at idx[first].  Returns the cut.
__device__ int sel_partition_warp(const SelView& v, int first, int last) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const double pk = v.key[v.idx[first]];
    int nG = 0;
    for (int base = first + 1; base < last; base += 32) {
        const int p = base + lane;
        const bool f = p < last && !(v.key[v.idx[p]] < pk);
        const unsigned b = __ballot_sync(0xffffffffu, f);
        if (f) v.G[nG + __popc(b & lt)] = p;
        nG += __popc(b);
    }
    int nL = 0;
    for (int top = last - 1; top >= first; top -= 32) {
        const int p = top - lane;
        const bool f = p >= first && !(pk < v.key[v.idx[p]]);
        const unsigned b = __ballot_sync(0xffffffffu, f);
        if (f) v.L[nL + __popc(b & lt)] = p;
        nL += __popc(b);
    }
    __syncwarp();
    const int lim = min(nG, nL);
    int nswap = 0;
    for (int base = 0; base < lim; base += 32) {
        const int t = base + lane;
        const bool f = t < lim && v.G[t] < v.L[t];
        nswap += __popc(__ballot_sync(0xffffffffu, f));
    }
    for (int t = lane; t < nswap; t += 32) {
        const int a = v.G[t], b = v.L[t];
        const int ia = v.idx[a], ib = v.idx[b];
        v.idx[a] = ib;
        v.idx[b] = ia;
    }
    const int gm = nswap < nG ? v.G[nswap] : INT_MAX;
    const int lm1 = nswap >= 1 ? v.L[nswap - 1] : INT_MAX;
    __syncwarp();
    return min(gm, lm1);
}

__device__ int sel_partition_pivot_warp(const SelView& v, int first, int last) {
    const int mid = first + (last - first) / 2;
    if ((threadIdx.x & 31) == 0) sel_move_median_to_first(v, first, first + 1, mid, last - 1);
    __syncwarp();
    return sel_partition_warp(v, first, last);
}

// std::nth_element(idx, idx + nth, idx + n)
__device__ void sel_nth_element_warp(const SelView& v, int n, int nth) {
    const int lane = threadIdx.x & 31;
    if (n == 0 || nth == n) return;
    int first = 0, last = n;
    int depth = lg_floor(n) * 2;
    while (last - first > 3) {
        if (depth == 0) {
            if (lane == 0) {
                sel_heap_select(v, first, nth + 1, last);
                const int t = v.idx[first]; v.idx[first] = v.idx[nth]; v.idx[nth] = t;
            }
            __syncwarp();
            return;
        }
        --depth;
        const int cut = sel_partition_pivot_warp(v, first, last);
        if (cut <= nth) first = cut;
        else last = cut;
    }
    if (lane == 0) sel_insertion_sort(v, first, last);
    __syncwarp();
}

// std::sort(idx, idx + k) for k <= 32
__device__ void sel_sort_small_warp(const SelView& v, int k) {
    const int lane = threadIdx.x & 31;
    if (k <= 1) return;
    if (k > 16) {
        // __introsort_loop with an explicit stack; ranges are disjoint, so the
        // processing order does not change the result.
        int sf[8], sl[8], sd[8], sp = 0;
        sf[0] = 0; sl[0] = k; sd[0] = lg_floor(k) * 2; sp = 1;
        while (sp > 0) {
            --sp;
            int f = sf[sp], l = sl[sp], d = sd[sp];
            while (l - f > 16) {
                if (d == 0) {
                    if (lane == 0) { sel_heap_select(v, f, l, l); sel_sort_heap(v, f, l); }
                    __syncwarp();
                    break;
                }
                --d;
                const int cut = sel_partition_pivot_warp(v, f, l);
                if (sp < 8) { sf[sp] = cut; sl[sp] = l; sd[sp] = d; ++sp; }
                l = cut;
            }
        }
    }
    // final insertion sort == stable sort of the current arrangement
    const int e = lane < k ? v.idx[lane] : 0;
    const double ke = lane < k ? v.key[e] : 0.0;
    int rank = 0;
    for (int m = 0; m < k; ++m) {
        const double km = __shfl_sync(0xffffffffu, ke, m);
        if (lane < k && (km < ke || (!(ke < km) && m < lane))) ++rank;
    }
    __syncwarp();
    if (lane < k) v.idx[rank] = e;
    __syncwarp();
}

// select_top_k_indices: indices 0..n-1 in v.idx, result in v.idx[0..k)
__device__ void sel_top_k_warp(const SelView& v, int n, int k) {
    const int lane = threadIdx.x & 31;
    for (int i = lane; i < n; i += 32) v.idx[i] = i;
    __syncwarp();
    if (n <= 0 || k <= 0) return;
    if (k < n) sel_nth_element_warp(v, n, k);
    sel_sort_small_warp(v, k);
}


// ---- CTA-level std::sort, first `keep` positions ---------------------------
// std::sort(first, last, comp) = __introsort_loop (depth limit 2 floor(lg n),
// ranges above 16 partitioned around a median-of-three pivot, heap sort of a
// range whose depth ran out) + __final_insertion_sort.  Every partition
// leaves [first, cut) <= pivot <= [cut, last), so the final insertion sort
// never moves an element out of its leaf range (it only passes strictly
// greater elements): it is a stable sort of each leaf.  Ranges are disjoint,
// so their processing order is free, and a range that starts at or beyond
// `keep` never changes a position below it: it is dropped.
//
// Ranges longer than kSortWarpRange are partitioned by the whole CTA (the
// data-parallel G/L form above, with ordered block compaction), shorter ones
// by one warp each in its shared-memory slab (keys, ids and G/L staged there).
constexpr int kSortWarpRange = 256;
constexpr int kSortStack = 64;
// per-warp slab: keys[256] f64 | pos->local[256] | local->id[256] | G[256] | L[264] | leaf mask[8]
constexpr int kSortSlabBytes = 2048 + 1024 + 1024 + 1024 + 1056 + 32;
__host__ __device__ constexpr int sort_smem_bytes(int warps) { return warps * kSortSlabBytes; }

struct SortRange { int f, l, d; };

// exclusive scan of one int per thread over the CTA; total -> *tot (shared)
__device__ __forceinline__ int blk_scan_excl1(int v, int* sh, int* tot) {
    const int t = threadIdx.x, lane = t & 31, w = t >> 5, nw = blockDim.x >> 5;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) { const int y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
    if (lane == 31) sh[w] = x;
    __syncthreads();
    int y = lane < nw ? sh[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) { const int z = __shfl_up_sync(0xffffffffu, y, o); if (lane >= o) y += z; }
    const int wbase = __shfl_sync(0xffffffffu, y, (w + 31) & 31);
    const int total = __shfl_sync(0xffffffffu, y, 31);
    if (t == 0) *tot = total;
    const int r = (w > 0 ? wbase : 0) + x - v;
    __syncthreads();
    return r;
}

// Hoare partition of [first+1, last) around idx[first] by the whole CTA;
// G and L are global scratch of last - first entries each.
__device__ int sel_partition_block(const SelView& v, int first, int last, int* sh) {
    const int T = blockDim.x, t = threadIdx.x;
    const double pk = v.key[v.idx[first]];
    // G: ascending positions of [first+1, last) with !(key < pivot)
    const int cg = (last - first - 1 + T - 1) / T;
    const int g0 = min(last, first + 1 + t * cg), g1 = min(last, g0 + cg);
    int ng = 0;
    for (int p = g0; p < g1; ++p) ng += !(v.key[v.idx[p]] < pk);
    int og = blk_scan_excl1(ng, sh, sh + 32);
    for (int p = g0; p < g1; ++p)
        if (!(v.key[v.idx[p]] < pk)) v.G[og++] = p;
    // L: descending positions of [first, last) with !(pivot < key)
    const int cl = (last - first + T - 1) / T;
    const int l1 = max(first, last - t * cl), l0 = max(first, l1 - cl);
    int nl = 0;
    for (int p = l1 - 1; p >= l0; --p) nl += !(pk < v.key[v.idx[p]]);
    int ol = blk_scan_excl1(nl, sh, sh + 33);
    for (int p = l1 - 1; p >= l0; --p)
        if (!(pk < v.key[v.idx[p]])) v.L[ol++] = p;
    __syncthreads();
    const int nG = sh[32], nL = sh[33];
    if (t == 0) {
        // G ascends and L descends, so G[t] < L[t] holds on a prefix
        int lo = 0, hi = min(nG, nL);
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (v.G[mid] < v.L[mid]) lo = mid + 1;
            else hi = mid;
        }
        sh[34] = lo;
    }
    __syncthreads();
    const int nswap = sh[34];
    for (int q = t; q < nswap; q += T) {
        const int a = v.G[q], b = v.L[q];
        const int ia = v.idx[a], ib = v.idx[b];
        v.idx[a] = ib;
        v.idx[b] = ia;
    }
    const int gm = nswap < nG ? v.G[nswap] : INT_MAX;
    const int lm1 = nswap >= 1 ? v.L[nswap - 1] : INT_MAX;
    __syncthreads();
    return min(gm, lm1);
}

// One warp: the introsort of range [f, l) (depth d) in its slab, then the
// stable sort of every leaf; positions at or beyond `keep` are not finished.
__device__ void sel_sort_range_warp(const SelView& g, SortRange r, int keep, unsigned char* slab) {
    const int lane = threadIdx.x & 31;
    const int m = r.l - r.f;
    double* skey = reinterpret_cast<double*>(slab);
    int* sidx = reinterpret_cast<int*>(slab + 2048);
    int* gid = sidx + 256;
    int* G = gid + 256;
    int* L = G + 256;
    unsigned* leaf = reinterpret_cast<unsigned*>(L + 264);
    for (int j = lane; j < m; j += 32) {
        const int e = g.idx[r.f + j];
        gid[j] = e;
        skey[j] = g.key[e];
        sidx[j] = j;
    }
    if (lane < 8) leaf[lane] = 0u;
    __syncwarp();
    const SelView v{sidx, skey, G, L};
    int sf[kSortStack], sl[kSortStack], sd[kSortStack], sp = 0;
    sf[0] = 0; sl[0] = m; sd[0] = r.d; sp = 1;
    while (sp > 0) {
        --sp;
        const int a = sf[sp];
        int b = sl[sp], d = sd[sp];
        while (true) {
            if (r.f + a >= keep || b - a <= 16) break;
            if (d == 0) {
                if (lane == 0) { sel_make_heap(v, a, b); sel_sort_heap(v, a, b); }
                __syncwarp();
                break;
            }
            --d;
            const int cut = sel_partition_pivot_warp(v, a, b);
            if (sp < kSortStack) { sf[sp] = cut; sl[sp] = b; sd[sp] = d; ++sp; }
            b = cut;
        }
        if (lane == 0) leaf[a >> 5] |= 1u << (a & 31);
        __syncwarp();
    }
    // stable sort of each leaf: rank = smaller keys + equal keys before
    for (int p = lane; p < m; p += 32) {
        int s = p;
        while (!((leaf[s >> 5] >> (s & 31)) & 1u)) --s;
        int e = p + 1;
        while (e < m && !((leaf[e >> 5] >> (e & 31)) & 1u)) ++e;
        const double kp = skey[sidx[p]];
        int rank = 0;
        for (int q = s; q < e; ++q) {
            const double kq = skey[sidx[q]];
            rank += (kq < kp || (!(kp < kq) && q < p)) ? 1 : 0;
        }
        G[s + rank] = sidx[p];
    }
    __syncwarp();
    for (int p = lane; p < m; p += 32) g.idx[r.f + p] = gid[G[p]];
    __syncwarp();
}

// std::sort(idx, idx + n) by key, exact in positions [0, keep).  The CTA
// calls it together; v.G and v.L hold n + 1 ints of global scratch, `small`
// room for keep + kSortWarpRange ranges, `slab` sort_smem_bytes(warps) of
// dynamic shared memory.
__device__ void sel_sort_prefix_block(const SelView& v, int n, int keep, SortRange* small, unsigned char* slab) {
    __shared__ int sh[40];
    __shared__ SortRange stk[kSortStack];
    __shared__ int sp, nsmall;
    __shared__ SortRange cur;
    if (threadIdx.x == 0) {
        stk[0] = SortRange{0, n, 2 * lg_floor(max(n, 1))};
        sp = 1;
        nsmall = 0;
    }
    while (true) {
        __syncthreads();
        const int top = sp;
        __syncthreads();          // every thread has read sp before thread 0 pops
        if (top == 0) break;
        if (threadIdx.x == 0) { cur = stk[top - 1]; sp = top - 1; }
        __syncthreads();
        SortRange r = cur;
        while (true) {
            if (r.f >= keep || r.l - r.f <= 1) break;
            if (r.l - r.f <= kSortWarpRange) {
                if (threadIdx.x == 0) small[nsmall++] = r;
                break;
            }
            if (r.d == 0) {
                if (threadIdx.x == 0) { sel_make_heap(v, r.f, r.l); sel_sort_heap(v, r.f, r.l); }
                break;
            }
            --r.d;
            if (threadIdx.x == 0) sel_move_median_to_first(v, r.f, r.f + 1, r.f + (r.l - r.f) / 2, r.l - 1);
            __syncthreads();
            const int cut = sel_partition_block(v, r.f, r.l, sh);
            if (threadIdx.x == 0 && sp < kSortStack) stk[sp++] = SortRange{cut, r.l, r.d};
            r.l = cut;
        }
    }
    const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int q = w; q < nsmall; q += nw) sel_sort_range_warp(v, small[q], keep, slab + (size_t)w * kSortSlabBytes);
    __syncthreads();
}

}  // namespace nx
