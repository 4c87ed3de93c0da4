// batch.cuh — one launch per kernel for many independent worlds.
//
// Every kernel of the step is a __device__ body plus a __global__ wrapper.
// For a batch, each world's step sequence is recorded instead of launched:
// per launch the body, the launch shape and the argument values packed into
// a Pack.  Worlds whose sequences name the same bodies in the same order form
// a group; the group then runs each position of its sequence as ONE launch of
// k_batched<body> with gridDim.y = number of worlds, whose blocks read their
// world's arguments from a device table (row blockIdx.y).  Per-world control
// flow that the host decided (adaptive barrier on/off, ALM iteration count)
// is part of the sequence, so worlds only share launches that they would all
// have made; data-dependent control flow stays on the device (the ALM and
// detection gates), exactly as for one world.
#pragma once

#include <cstring>
#include <type_traits>
#include <vector>

#include <cuda_runtime.h>

namespace nx {

template <typename T> struct ident { using type = T; };

template <typename... A> struct Pack;
template <> struct Pack<> {};
template <typename H, typename... T> struct Pack<H, T...> {
    H h;
    Pack<T...> t;
};

template <typename... A> Pack<A...> make_pack(A... a);
template <typename H, typename... T> Pack<H, T...> make_pack_impl(H h, T... t) {
    Pack<H, T...> p;
    p.h = h;
    p.t = make_pack<T...>(t...);
    return p;
}
template <typename... A> Pack<A...> make_pack(A... a) {
    if constexpr (sizeof...(A) == 0) return Pack<>{};
    else return make_pack_impl<A...>(a...);
}

// Calls F with the packed values, each bound by reference to the table row.
template <auto F, typename P, typename... D>
__device__ __forceinline__ void call_packed(const P& p, const D&... d) {
    if constexpr (std::is_same_v<P, Pack<>>) F(d...);
    else call_packed<F>(p.t, d..., p.h);
}

template <auto F, typename P>
__global__ void k_batched(const P* __restrict__ tab) { call_packed<F>(tab[blockIdx.y]); }
template <auto F, int LB, typename P>
__global__ void __launch_bounds__(LB) k_batched_lb(const P* __restrict__ tab) { call_packed<F>(tab[blockIdx.y]); }

// ---------------------------------------------------------------------------
// Queue form for kernels whose work per world is known only on the device
// (the narrow phase: the world's body-pair count).  Work items are (world,
// chunk) pairs: a preparation block counts each world's chunks (ITEMS) and
// forms their prefix over worlds; a persistent grid then pulls item numbers
// from a counter, finds the item's world by binary search over the prefix,
// and runs the body as block `chunk` of a grid of that world's chunk count.
// Each item writes only its own world's outputs at fixed places, so the
// result does not depend on which block takes which item.
// ---------------------------------------------------------------------------
template <auto ITEMS, typename P, typename... D>
__device__ __forceinline__ int items_packed(const P& p, const D&... d) {
    if constexpr (std::is_same_v<P, Pack<>>) return ITEMS(d...);
    else return items_packed<ITEMS>(p.t, d..., p.h);
}
template <auto F, typename P, typename... D>
__device__ __forceinline__ void call_packed_v(const P& p, int vb, int vg, const D&... d) {
    if constexpr (std::is_same_v<P, Pack<>>) F(d..., vb, vg);
    else call_packed_v<F>(p.t, vb, vg, d..., p.h);
}

constexpr int kQueuePrepThreads = 1024;

// prefix[0..nw] of the worlds' item counts (one block), counter = 0
template <auto ITEMS, typename P>
__global__ void __launch_bounds__(kQueuePrepThreads) k_queue_prep(const P* __restrict__ tab, int nw, int* prefix, int* counter) {
    __shared__ int warp_tot[kQueuePrepThreads / 32];
    __shared__ int carry;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (threadIdx.x == 0) { carry = 0; prefix[0] = 0; *counter = 0; }
    __syncthreads();
    for (int base = 0; base < nw; base += kQueuePrepThreads) {
        const int w = base + threadIdx.x;
        const int v = w < nw ? items_packed<ITEMS>(tab[w]) : 0;
        int x = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_tot[wid] = x;
        __syncthreads();
        if (wid == 0) {
            int t = warp_tot[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            warp_tot[lane] = t;   // inclusive over warps
        }
        __syncthreads();
        const int incl = carry + (wid ? warp_tot[wid - 1] : 0) + x;
        if (w < nw) prefix[w + 1] = incl;
        __syncthreads();
        if (threadIdx.x == kQueuePrepThreads - 1) carry = incl;
        __syncthreads();
    }
}

template <auto F, int LB, typename P>
__global__ void __launch_bounds__(LB) k_batched_queue(const P* __restrict__ tab, int nw, const int* __restrict__ prefix,
                                                      int* counter) {
    __shared__ int item;
    const int total = prefix[nw];
    for (;;) {
        if (threadIdx.x == 0) item = atomicAdd(counter, 1);
        __syncthreads();
        const int it = item;
        if (it >= total) return;
        int lo = 0, hi = nw - 1;   // the last world whose prefix is <= it
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (prefix[mid] <= it) lo = mid;
            else hi = mid - 1;
        }
        call_packed_v<F>(tab[lo], it - prefix[lo], prefix[lo + 1] - prefix[lo]);
        __syncthreads();           // `item` is rewritten on the next trip
    }
}

// One recorded launch of one world.
struct LaunchRec {
    const void* kern;                 // host stub of k_batched<body, ...> (or k_batched_queue)
    const void* prep = nullptr;       // k_queue_prep of a queue-form launch
    int queue_kind = -1;              // which queue-form kernel (its persistent grid is tunable)
    dim3 grid, block;
    size_t smem;
    int fam;
    size_t align;
    std::vector<unsigned char> args;  // the Pack of this world's argument values
};

template <auto F, int LB, typename... P>
void record_into(std::vector<LaunchRec>& out, int fam, void (*)(P...), dim3 g, dim3 b, size_t smem,
                 typename ident<std::decay_t<P>>::type... args) {
    using PK = Pack<std::decay_t<P>...>;
    const PK pk = make_pack<std::decay_t<P>...>(args...);
    LaunchRec r;
    if constexpr (LB > 0) r.kern = (const void*)&k_batched_lb<F, LB, PK>;
    else r.kern = (const void*)&k_batched<F, PK>;
    r.grid = g; r.block = b; r.smem = smem; r.fam = fam; r.align = alignof(PK);
    r.args.resize(sizeof(PK));
    std::memcpy(r.args.data(), &pk, sizeof(PK));
    out.push_back(std::move(r));
}

}  // namespace nx

namespace nx {

// a queue-form launch: parameter types from the item counter's signature
// (the body's parameters without the trailing block index and count)
template <auto F, auto ITEMS, int LB, typename... P>
void record_queue_into(std::vector<LaunchRec>& out, int fam, int queue_kind, int (*)(P...), dim3 g, dim3 b, size_t smem,
                       typename ident<std::decay_t<P>>::type... args) {
    using PK = Pack<std::decay_t<P>...>;
    const PK pk = make_pack<std::decay_t<P>...>(args...);
    LaunchRec r;
    r.kern = (const void*)&k_batched_queue<F, LB, PK>;
    r.prep = (const void*)&k_queue_prep<ITEMS, PK>;
    r.queue_kind = queue_kind;
    r.grid = g; r.block = b; r.smem = smem; r.fam = fam; r.align = alignof(PK);
    r.args.resize(sizeof(PK));
    std::memcpy(r.args.data(), &pk, sizeof(PK));
    out.push_back(std::move(r));
}

}  // namespace nx
