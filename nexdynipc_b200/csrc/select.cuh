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

}  // namespace nx
