// pcg.cuh — block-Jacobi preconditioned conjugate gradients over a 6x6-block
// BSR matrix, the whole solve in one cooperative-grid kernel.
//
// The iteration (x0 = 0, r = b, z = M^-1 r, p = z):
//   q = A p;  alpha = (r.z) / (p.q);  r' = r - alpha q;  z' = M^-1 r';
//   beta = (r'.z') / (r.z);  x += alpha p;  p' = z' + beta p
// with M the block diagonal of A.  r' and z' are formed inside the reduction
// that needs them (z' stored there, r' formed again with the same arithmetic
// in the update) and p.q is summed in the product's own pass, so an iteration
// crosses three grid barriers: in the p.q sum, in the joint (r'.r', r'.z')
// sum, after the update (r, p double-buffered).  The product is the HBM-bound part: one thread per
// row component reads its row's 48-byte slices of every block in the row.
// Sums use a fixed-order grid reduction over coalesced reads, so results do
// not depend on timing.
#pragma once

namespace nx {

struct PcgArgs {
    int N;
    const int* rp; const int* ci; const double* vals;   // BSR, 36 doubles per block
    const double* minv;                                 // [36N] inverse diagonal blocks
    const double* b;
    double* x;
    double* r[2]; double* p[2]; double* q; double* z;
    double tol; int max_iter;
    double* part; int stride;                           // grid partial sums, 2 * kRedMaxQ * stride
    unsigned* bar_count; int* bar_abort; int* status;
    int* iters_out; double* res_out;                    // iterations, final |r| / |b|
};

// summed diagonal blocks (storage order) and their inverses by 6x6 LDL^T
__global__ void k_pcg_prepare(int N, const int* rp, const int* ci, const double* vals, double* minv, int* fail) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double A0[36];
    for (int e = 0; e < 36; ++e) A0[e] = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k)
        if (ci[k] == i)
            for (int e = 0; e < 36; ++e) A0[e] += vals[36LL * k + e];
    for (int c = 0; c < 6; ++c) {
        double A[36], u[6];
        for (int e = 0; e < 36; ++e) A[e] = A0[e];
        for (int e = 0; e < 6; ++e) u[e] = e == c ? 1.0 : 0.0;
        if (!ldlt6_solve(A, u)) { atomicExch(fail, 1); return; }
        for (int e = 0; e < 6; ++e) minv[36LL * i + 6 * e + c] = u[e];
    }
}

// row component e of A p: the row's 48-byte slice of each block read as three
// 16-byte read-only loads (block offsets are multiples of 288 B and slice
// offsets of 48 B, so every load is 16-byte aligned)
__device__ __forceinline__ double pcg_row_product(const PcgArgs& A, const double* p, int e) {
    const int i = e / 6, rr = e % 6;
    const int k0 = __ldg(A.rp + i), k1 = __ldg(A.rp + i + 1);
    double acc = 0.0;
    auto slice = [&](int k) {
        const double2* blk = reinterpret_cast<const double2*>(A.vals + 36LL * k + 6 * rr);
        const double2 a0 = __ldg(blk), a1 = __ldg(blk + 1), a2 = __ldg(blk + 2);
        const double2* pc = reinterpret_cast<const double2*>(p + 6LL * __ldg(A.ci + k));
        const double2 b0 = pc[0], b1 = pc[1], b2 = pc[2];
        double t = 0.0;
        t += a0.x * b0.x; t += a0.y * b0.y; t += a1.x * b1.x;
        t += a1.y * b1.y; t += a2.x * b2.x; t += a2.y * b2.y;
        return t;
    };
    int k = k0;
    // two blocks per trip: both blocks' loads are in flight together; the
    // partial products still enter acc in block order
    for (; k + 1 < k1; k += 2) {
        const double t0 = slice(k), t1 = slice(k + 1);
        acc += t0;
        acc += t1;
    }
    if (k < k1) acc += slice(k);
    return acc;
}
// component e of M^-1 (r - alpha q)
__device__ __forceinline__ double pcg_precond(const PcgArgs& A, const double* r, const double* q, double alpha, int e) {
    const int i = e / 6, rr = e % 6;
    const double* m = A.minv + 36LL * i + 6 * rr;
    double t = 0.0;
#pragma unroll
    for (int c = 0; c < 6; ++c) t += m[c] * (r[6 * i + c] - alpha * q[6 * i + c]);
    return t;
}

constexpr int kPcgThreads = 512;
constexpr int kPcgMaxQ = 2;   // sums per reduction call

// Grid sums with coalesced reads: thread t folds elements t, t + T, ...
// (T threads in the grid), then a shuffle-down tree per warp, a tree over
// the CTA's warps, one partial per CTA, a grid barrier, and every thread
// folds the G partials the same way.  Deterministic for a given grid.
template <int Q>
__device__ void pcg_grid_fold(GridCtx& gc, double* sh, double* part, int& parity, const double (&acc)[Q], double (&out)[Q]);

template <int Q, typename F>
__device__ void pcg_sums(GridCtx& gc, double* sh, double* part, int& parity, int n, F f, double (&out)[Q]) {
    double acc[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) acc[q] = 0.0;
    for (int e = gc.gtid; e < n; e += gc.gthreads)
#pragma unroll
        for (int q = 0; q < Q; ++q) acc[q] += f(q, e);
    pcg_grid_fold<Q>(gc, sh, part, parity, acc, out);
}

// the grid part of pcg_sums, from each thread's running sums (includes one
// grid barrier, so every write made before it is visible after it)
template <int Q>
__device__ void pcg_grid_fold(GridCtx& gc, double* sh, double* part, int& parity, const double (&acc)[Q], double (&out)[Q]) {
    const unsigned full = 0xffffffffu;
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
    // two alternating slots of a fixed size, so that a call's partials never
    // overwrite those of the previous call while a CTA may still fold them
    static_assert(Q <= kPcgMaxQ, "too many simultaneous sums");
    double* gp = part + (size_t)parity * kPcgMaxQ * gc.G;
    parity ^= 1;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        double v = acc[q];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(full, v, o);
        if (l == 0) sh[q * 32 + w] = v;
    }
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            double v = l < nw ? sh[q * 32 + l] : 0.0;
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(full, v, o);
            if (l == 0) gp[q * gc.G + gc.b] = v;
        }
    }
    gc.sync();
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        double v = 0.0;
        for (int e = l; e < gc.G; e += 32) v += __ldcg(gp + q * gc.G + e);
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(full, v, o);
        out[q] = __shfl_sync(full, v, 0);
    }
}

__global__ void __launch_bounds__(kPcgThreads) k_pcg(const __grid_constant__ PcgArgs A) {
    __shared__ double sh_red[kRedMaxQ * 32];
    __shared__ int sh_ok;
    if (threadIdx.x == 0) sh_ok = 1;
    GridCtx gc;
    gc.G = gridDim.x; gc.b = blockIdx.x;
    gc.gtid = blockIdx.x * blockDim.x + threadIdx.x; gc.gthreads = gridDim.x * blockDim.x;
    gc.lin = gc.gtid;
    gc.count = A.bar_count; gc.abort = A.bar_abort; gc.status = A.status; gc.target = 0; gc.sh_ok = &sh_ok;
    gc.cluster = false; gc.limit = kBarrierSpinLimit;
    __syncthreads();
    int parity = 0;
    const int n = 6 * A.N;
    // x = 0, r = b, p = M^-1 b
    for (int e = gc.gtid; e < n; e += gc.gthreads) {
        A.x[e] = 0.0;
        A.r[0][e] = A.b[e];
        A.p[0][e] = pcg_precond(A, A.b, A.b, 0.0, e);
    }
    if (!gc.sync()) return;
    double init[2];
    pcg_sums<2>(gc, sh_red, A.part, parity, n, [&](int qq, int e) { return qq == 0 ? A.b[e] * A.b[e] : A.r[0][e] * A.p[0][e]; },
                init);
    const double bnorm = sqrt(init[0]);
    double rz = init[1];
    int it = 0, cur = 0;
    double res = bnorm > 0.0 ? 1.0 : 0.0;
    while (it < A.max_iter && res > A.tol) {
        const double* p = A.p[cur];
        const double* r = A.r[cur];
        // Ap and p.Ap in one pass (the fold's grid barrier publishes Ap)
        double pqa[1] = {0.0}, pqv[1];
        for (int e = gc.gtid; e < n; e += gc.gthreads) {
            const double qe = pcg_row_product(A, p, e);
            A.q[e] = qe;
            pqa[0] += p[e] * qe;
        }
        pcg_grid_fold<1>(gc, sh_red, A.part, parity, pqa, pqv);
        if (!*gc.sh_ok) return;
        const double pq = pqv[0];
        if (!(pq > 0.0)) { if (gc.gtid == 0) atomicExch(A.status, NXD_FACTOR_FAILED); break; }
        const double alpha = rz / pq;
        double s2[2];
        pcg_sums<2>(gc, sh_red, A.part, parity, n, [&](int qq, int e) {
            const double rn = r[e] - alpha * A.q[e];
            if (qq == 0) return rn * rn;
            const double zz = pcg_precond(A, r, A.q, alpha, e);
            A.z[e] = zz;                    // kept for the update: one read of M^-1 per iteration
            return rn * zz;
        }, s2);
        const double beta = s2[1] / rz;
        rz = s2[1];
        double* rn = A.r[cur ^ 1];
        double* pn = A.p[cur ^ 1];
        for (int e = gc.gtid; e < n; e += gc.gthreads) {
            A.x[e] += alpha * p[e];
            rn[e] = r[e] - alpha * A.q[e];
            pn[e] = A.z[e] + beta * p[e];
        }
        if (!gc.sync()) return;
        cur ^= 1;
        ++it;
        res = bnorm > 0.0 ? sqrt(s2[0]) / bnorm : 0.0;
    }
    if (gc.gtid == 0) { *A.iters_out = it; *A.res_out = res; }
}

}  // namespace nx
