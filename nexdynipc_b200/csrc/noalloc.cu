// noalloc.cu — body-pair broad phase that allocates nothing.
//
// Some callers cannot call cudaMalloc: an engine that hands every device
// byte out of its own pool, a process running under a hard memory cap or a
// real-time loop that forbids allocator calls after start-up.  They own the
// input and output buffers and pass them in; everything else this entry
// point needs lives in the fixed scratch array below, which every GPU that
// loads the library keeps until the process exits.
//
// Result: the same pairs, in the same order, as nxd_body_pairs (the
// reference's ContactAssembler::detectBodyPairs on the current poses), given
// each body's local box -- an empty one (min > max) for a body without a mesh.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/nxd.h"
#include "nx_math.cuh"

using namespace nx;

namespace {

constexpr int kMaxBodies = NXD_NOALLOC_MAX_BODIES;
// scratch layout: world boxes [kMaxBodies*6] doubles, then per-body pair
// counts, exclusive offsets [kMaxBodies] ints each, then the total.
constexpr size_t kBoxBytes = sizeof(double) * 6 * kMaxBodies;
constexpr size_t kScratchBytes = kBoxBytes + sizeof(int) * (2 * kMaxBodies + 32);

}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

struct Scratch {
    double* boxes;
    int* counts;
    int* offsets;
    int* total;
};

Scratch carve(unsigned char* base) {
    Scratch s;
    s.boxes = reinterpret_cast<double*>(base);
    s.counts = reinterpret_cast<int*>(base + kBoxBytes);
    s.offsets = s.counts + kMaxBodies;
    s.total = s.offsets + kMaxBodies;
    return s;
}

// Device address of the scratch array, looked up once per device with that
// device current (the symbol's host-side name is only a stand-in).
std::mutex g_mu;
unsigned char* g_addr[64] = {};

nxd_status scratch_for_current_device(Scratch* out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return NXD_NO_DEVICE;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            std::fprintf(stderr, "nxd_body_pairs_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
            return NXD_CUDA_ERROR;
        }
        g_addr[dev] = static_cast<unsigned char*>(p);
    }
    *out = carve(g_addr[dev]);
    return NXD_OK;
}

// A local box with min > max on some axis (or a NaN) marks a body without a
// mesh: nxd_body_pairs leaves such bodies out of every pair, so its world box
// is stored as NaNs, which fail every overlap test at any inflation.
__global__ void k_na_boxes(const double* pos, const double* quat, const double* lbox, int n, double* boxes) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const V3 lo = ld3(lbox + 6 * i), hi = ld3(lbox + 6 * i + 3);
    if (!(lo.x <= hi.x && lo.y <= hi.y && lo.z <= hi.z)) {
        const double q = __longlong_as_double(0x7ff8000000000000LL);
        for (int k = 0; k < 6; ++k) boxes[6 * i + k] = q;
        return;
    }
    const Box b = transform_local_box(lo, hi, ld3(pos + 3 * i), ldq(quat + 4 * i));
    st3(boxes + 6 * i, b.mn);
    st3(boxes + 6 * i + 3, b.mx);
}

__device__ __forceinline__ bool na_overlap(const double* boxes, int i, int j, double m) {
    Box a, b;
    a.mn = ld3(boxes + 6 * i); a.mx = ld3(boxes + 6 * i + 3);
    b.mn = ld3(boxes + 6 * j); b.mx = ld3(boxes + 6 * j + 3);
    return box_intersects(box_inflated(a, m), box_inflated(b, m));
}

// one warp per i; j scanned from n-1 down (the reference's BVH reports the
// overlapping j > i in descending order)
__global__ void k_na_pairs(const double* boxes, int n, double r, int* counts, const int* offsets, int* out, long long cap) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const double m = dmax(0.0, r);
    const unsigned lt = (1u << lane) - 1u;
    for (int i = warp; i < n; i += nw) {
        int c = 0;
        const int base = out ? offsets[i] : 0;
        for (int top = n - 1; top > i; top -= 32) {
            const int j = top - lane;
            const bool f = j > i && na_overlap(boxes, i, j, m);
            const unsigned b = __ballot_sync(0xffffffffu, f);
            if (out && f) {
                const long long pos = (long long)base + c + __popc(b & lt);
                if (pos < cap) { out[2 * pos] = i; out[2 * pos + 1] = j; }
            }
            c += __popc(b);
        }
        if (!out && lane == 0) counts[i] = c;
    }
}

// exclusive scan of counts[0..n) into offsets, total -> *total (one block)
__global__ void k_na_scan(const int* counts, int* offsets, int n, int* total) {
    __shared__ int part[1024];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < n; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const int v = i < n ? counts[i] : 0;
        part[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < (int)blockDim.x; o <<= 1) {
            const int y = threadIdx.x >= (unsigned)o ? part[threadIdx.x - o] : 0;
            __syncthreads();
            part[threadIdx.x] += y;
            __syncthreads();
        }
        if (i < n) offsets[i] = carry + part[threadIdx.x] - v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry += part[threadIdx.x];
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

}  // namespace

extern "C" nxd_status nxd_body_pairs_noalloc(const double* position, const double* orientation, const double* local_box,
                                             int32_t n, double inflation_radius, int32_t* pairs, int64_t cap,
                                             int64_t* count, void* stream) {
    if (n < 0 || !count || (n > 0 && (!position || !orientation || !local_box)) || (cap > 0 && !pairs))
        return NXD_INVALID_ARGUMENT;
    if (n > kMaxBodies) {
        std::fprintf(stderr, "nxd_body_pairs_noalloc: %d bodies exceed the fixed scratch limit of %d\n", n, kMaxBodies);
        return NXD_INVALID_ARGUMENT;
    }
    Scratch s;
    const nxd_status st = scratch_for_current_device(&s);
    if (st != NXD_OK) return st;
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    *count = 0;
    if (n < 2) return NXD_OK;
    // the total is the only scratch value read back; start it at zero
    if (cudaMemsetAsync(s.total, 0, sizeof(int), cs) != cudaSuccess) return NXD_CUDA_ERROR;
    k_na_boxes<<<(n + 127) / 128, 128, 0, cs>>>(position, orientation, local_box, n, s.boxes);
    const int blocks = (int)(((long long)n * 32 + 255) / 256);
    k_na_pairs<<<blocks, 256, 0, cs>>>(s.boxes, n, inflation_radius, s.counts, nullptr, nullptr, 0);
    k_na_scan<<<1, 1024, 0, cs>>>(s.counts, s.offsets, n, s.total);
    k_na_pairs<<<blocks, 256, 0, cs>>>(s.boxes, n, inflation_radius, nullptr, s.offsets, pairs, cap);
    int total = 0;
    if (cudaMemcpyAsync(&total, s.total, sizeof(int), cudaMemcpyDeviceToHost, cs) != cudaSuccess) return NXD_CUDA_ERROR;
    if (cudaStreamSynchronize(cs) != cudaSuccess) return NXD_CUDA_ERROR;
    *count = total;
    return total > cap ? NXD_CAPACITY : NXD_OK;
}
