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

// The matrix is symmetric, so the iteration reads its upper block triangle
// only (as LAPACK's uplo = 'U' solvers do): the diagonal blocks as their 21
// upper entries, each off-diagonal block (i, j), j > i, once -- row i reads
// its row slices, row j its column slices (A_ji = A_ij^T) -- which halves the
// bytes of the product.  The inverse diagonal blocks (symmetric too) are
// stored as 21 entries as well.  Duplicate blocks of the caller's BSR are
// summed (in storage order) when the triangle is built.
constexpr int kSym = 21;
// index of entry (r, c) in the packed upper triangle, rows in order
__host__ __device__ __forceinline__ int sym_at(int r, int c) {
    const int a = r < c ? r : c, b = r < c ? c : r;
    return a * 6 - (a * (a - 1)) / 2 + (b - a);
}

struct PcgArgs {
    int N;
    const int* urp; const int* uci; const double* uvals;  // upper off-diagonal blocks, 36 doubles each
    const int* lrp; const int* lidx; const int* lrow;     // per row j: the upper blocks (i, j), i < j
    const double* dsym;                                   // [21N] diagonal blocks, upper triangles
    const double* minv;                                   // [21N] inverse diagonal blocks
    const double* b;
    double* x;
    double* r[2]; double* p[2]; double* q; double* z;
    double tol; int max_iter;
    double* part; int stride;                           // grid partial sums, 2 * kRedMaxQ * stride
    unsigned* bar_count; int* bar_abort; int* status;
    int* iters_out; double* res_out;                    // iterations, final |r| / |b|
};

// summed diagonal blocks (storage order) and their inverses by 6x6 LDL^T
__global__ void k_pcg_prepare(int N, const int* rp, const int* ci, const double* vals, double* minv, double* dsym, int* fail) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double A0[36];
    for (int e = 0; e < 36; ++e) A0[e] = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k)
        if (ci[k] == i)
            for (int e = 0; e < 36; ++e) A0[e] += vals[36LL * k + e];
    for (int r = 0; r < 6; ++r)
        for (int c = r; c < 6; ++c) {
            dsym[(size_t)kSym * i + sym_at(r, c)] = A0[6 * r + c];
            A0[6 * c + r] = A0[6 * r + c];   // the factorisation sees the upper triangle only
        }
    double Mi[36];
    for (int c = 0; c < 6; ++c) {
        double A[36], u[6];
        for (int e = 0; e < 36; ++e) A[e] = A0[e];
        for (int e = 0; e < 6; ++e) u[e] = e == c ? 1.0 : 0.0;
        if (!ldlt6_solve(A, u)) { atomicExch(fail, 1); return; }
        for (int e = 0; e < 6; ++e) Mi[6 * e + c] = u[e];
    }
    for (int r = 0; r < 6; ++r)
        for (int c = r; c < 6; ++c) minv[(size_t)kSym * i + sym_at(r, c)] = Mi[6 * r + c];
}

// Per row: distinct columns above (ucnt) and below (lcnt) the diagonal.  A
// column counts at its first occurrence in the row's storage order.
__device__ __forceinline__ bool first_in_row(const int* ci, int k0, int k) {
    for (int t = k0; t < k; ++t)
        if (ci[t] == ci[k]) return false;
    return true;
}
__global__ void k_pcg_tri_count(int N, const int* rp, const int* ci, int* ucnt, int* lcnt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        int u = 0, l = 0;
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            if (ci[k] == i || !first_in_row(ci, rp[i], k)) continue;
            if (ci[k] > i) ++u;
            else ++l;
        }
        ucnt[i] = u;
        lcnt[i] = l;
    }
}
// the next distinct column of row i above `after` (INT_MAX when none)
__device__ __forceinline__ int next_col(const int* ci, int k0, int k1, int after) {
    int best = 0x7fffffff;
    for (int k = k0; k < k1; ++k)
        if (ci[k] > after && ci[k] < best) best = ci[k];
    return best;
}
// upper blocks of row i in ascending column order, duplicates summed
__global__ void k_pcg_tri_upper(int N, const int* rp, const int* ci, const double* vals, const int* urp, int* uci,
                                double* uvals) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const int k0 = rp[i], k1 = rp[i + 1];
        int col = i, slot = urp[i];
        for (;;) {
            col = next_col(ci, k0, k1, col);
            if (col == 0x7fffffff) break;
            double acc[36];
            for (int e = 0; e < 36; ++e) acc[e] = 0.0;
            for (int k = k0; k < k1; ++k)
                if (ci[k] == col)
                    for (int e = 0; e < 36; ++e) acc[e] += vals[36LL * k + e];
            uci[slot] = col;
            for (int e = 0; e < 36; ++e) uvals[36LL * slot + e] = acc[e];
            ++slot;
        }
    }
}
// row j's blocks below the diagonal, ascending: the stored upper block
// (i, j) of each, found in row i's sorted upper columns.  A block with no
// stored transpose (a structurally unsymmetric matrix) sets *fail.
__global__ void k_pcg_tri_lower(int N, const int* rp, const int* ci, const int* urp, const int* uci, const int* lrp,
                                int* lidx, int* lrow, int* fail) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < N; j += gridDim.x * blockDim.x) {
        const int k0 = rp[j], k1 = rp[j + 1];
        int col = -1, slot = lrp[j];
        for (;;) {
            col = next_col(ci, k0, k1, col);
            if (col >= j) break;
            int lo = urp[col], hi = urp[col + 1];
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (uci[mid] < j) lo = mid + 1;
                else hi = mid;
            }
            if (lo >= urp[col + 1] || uci[lo] != j) { atomicExch(fail, 1); lidx[slot] = -1; }
            else lidx[slot] = lo;
            lrow[slot] = col;
            ++slot;
        }
    }
}

// row component e of A p, in ascending column order: the blocks below the
// diagonal (column slices of their stored transposes), the diagonal block,
// the blocks above (row slices as three 16-byte loads: block offsets are
// multiples of 288 B and slice offsets of 48 B)
__device__ __forceinline__ double pcg_row_product(const PcgArgs& A, const double* p, int e) {
    const int j = e / 6, rr = e % 6;
    double acc = 0.0;
    auto column = [&](int s) {
        const double* blk = A.uvals + 36LL * __ldg(A.lidx + s);
        const double* pc = p + 6LL * __ldg(A.lrow + s);
        double t = 0.0;
#pragma unroll
        for (int c = 0; c < 6; ++c) t += __ldg(blk + 6 * c + rr) * pc[c];
        return t;
    };
    {
        const int s1 = __ldg(A.lrp + j + 1);
        int s = __ldg(A.lrp + j);
        for (; s + 1 < s1; s += 2) {   // two blocks in flight, added in order
            const double t0 = column(s), t1 = column(s + 1);
            acc += t0;
            acc += t1;
        }
        if (s < s1) acc += column(s);
    }
    {
        const double* d = A.dsym + (size_t)kSym * j;
        const double* pc = p + 6LL * j;
        double t = 0.0;
#pragma unroll
        for (int c = 0; c < 6; ++c) t += __ldg(d + sym_at(rr, c)) * pc[c];
        acc += t;
    }
    auto slice = [&](int k) {
        const double2* blk = reinterpret_cast<const double2*>(A.uvals + 36LL * k + 6 * rr);
        const double2 a0 = __ldg(blk), a1 = __ldg(blk + 1), a2 = __ldg(blk + 2);
        const double2* pc = reinterpret_cast<const double2*>(p + 6LL * __ldg(A.uci + k));
        const double2 b0 = pc[0], b1 = pc[1], b2 = pc[2];
        double t = 0.0;
        t += a0.x * b0.x; t += a0.y * b0.y; t += a1.x * b1.x;
        t += a1.y * b1.y; t += a2.x * b2.x; t += a2.y * b2.y;
        return t;
    };
    const int k1 = __ldg(A.urp + j + 1);
    int k = __ldg(A.urp + j);
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
    const double* m = A.minv + (size_t)kSym * i;
    double t = 0.0;
#pragma unroll
    for (int c = 0; c < 6; ++c) t += m[sym_at(rr, c)] * (r[6 * i + c] - alpha * q[6 * i + c]);
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
