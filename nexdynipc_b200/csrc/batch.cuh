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

// One recorded launch of one world.
struct LaunchRec {
    const void* kern;                 // host stub of k_batched<body, ...>
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
