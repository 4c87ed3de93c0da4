// ipc_cpu.cpp — CPU checker for the primitive-level contact model (full IPC).
//
// Test infrastructure, like refcpu.cpp: only tests/ and bench.py's CPU leg
// load it.  The reference has no primitive-level model, so this restates
// the published method (Li et al. 2020 IPC; Li et al. 2021 additive CCD)
// with the per-pair arithmetic shared with the kernels (ipc_pair.h), and
// checks everything around it independently:
//   - candidate sets by an exact uniform-grid search over the boxes (no BVH);
//   - the subspace PSD projection against a full 12x12 Jacobi projection
//     of the raw pair Hessian (nxo_ipc_pair);
//   - derivatives by finite differences (in tests/).
// Sums follow the device's fixed orders: energies through the padded
// pairwise tree, gradients and Hessian blocks in pair order.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <vector>

#include "refcpu.h"
#include "../nexdynipc_b200/csrc/ipc_pair.h"

using nx::V3;
namespace ipc = nx::ipc;

namespace {

struct Geo {
    int64_t nv = 0, nf = 0, ne = 0;
    int N = 0;
    std::vector<int32_t> vbody, fbody, fvert, ebody, evert;
    std::vector<double> wv, wv1, pos;
    std::vector<double> theta;   // [3N] rotation vectors of the iterate (zeros without one)
    // with dx: the arc motion (body-local vertices, orientations, x, dx) and
    // each body's swept-box pad (ipc::arc_box_pad)
    std::vector<double> vloc, quat, x, dx, pad;
};

Geo load(nxo_world* w, const double* x, const double* dx) {
    Geo g;
    nxo_prim_counts(w, &g.nv, &g.nf, &g.ne);
    g.N = nxo_body_count(w);
    g.vbody.resize(g.nv); g.fbody.resize(g.nf); g.fvert.resize(3 * g.nf); g.ebody.resize(g.ne); g.evert.resize(2 * g.ne);
    nxo_prim_topology(w, g.vbody.data(), g.fbody.data(), g.fvert.data(), g.ebody.data(), g.evert.data());
    g.wv.resize(3 * g.nv); g.pos.resize(3 * g.N);
    nxo_world_vertices_at(w, x, g.wv.data(), g.pos.data());
    g.theta.assign(3 * (size_t)g.N, 0.0);
    if (x)
        for (int b = 0; b < g.N; ++b)
            for (int k = 0; k < 3; ++k) g.theta[3 * b + k] = x[6 * b + 3 + k];
    if (dx) {
        std::vector<double> x1(6 * (size_t)g.N);
        for (size_t i = 0; i < x1.size(); ++i) x1[i] = x[i] + dx[i];
        g.wv1.resize(3 * g.nv);
        nxo_world_vertices_at(w, x1.data(), g.wv1.data(), nullptr);
        g.vloc.resize(3 * g.nv); g.quat.resize(4 * (size_t)g.N);
        nxo_local_vertices(w, g.vloc.data(), g.quat.data());
        g.x.assign(x, x + 6 * (size_t)g.N);
        g.dx.assign(dx, dx + 6 * (size_t)g.N);
        std::vector<double> rmax(g.N, 0.0);
        for (int64_t v = 0; v < g.nv; ++v)
            rmax[g.vbody[v]] = nx::dmax(rmax[g.vbody[v]], nx::norm(nx::ld3(&g.vloc[3 * v])));
        g.pad.resize(g.N);
        for (int b = 0; b < g.N; ++b) g.pad[b] = ipc::arc_box_pad(nx::ld3(&g.dx[6 * b + 3]), rmax[b]);
    }
    return g;
}

struct Box { double mn[3], mx[3]; };

Box box_of(const Geo& g, const int32_t* vid, int nvid, double infl, int body) {
    if (!g.pad.empty()) infl = infl + g.pad[body];
    V3 mn = nx::ld3(&g.wv[3 * vid[0]]), mx = mn;
    for (int k = 0; k < nvid; ++k) {
        const V3 a = nx::ld3(&g.wv[3 * vid[k]]);
        mn = nx::cwmin(mn, a); mx = nx::cwmax(mx, a);
        if (!g.wv1.empty()) { const V3 b = nx::ld3(&g.wv1[3 * vid[k]]); mn = nx::cwmin(mn, b); mx = nx::cwmax(mx, b); }
    }
    const V3 e = nx::v3(infl, infl, infl);
    const V3 lo = mn - e, hi = mx + e;
    return Box{{lo.x, lo.y, lo.z}, {hi.x, hi.y, hi.z}};
}

bool overlap(const Box& a, const Box& b) {
    return a.mn[0] <= b.mx[0] && b.mn[0] <= a.mx[0] && a.mn[1] <= b.mx[1] && b.mn[1] <= a.mx[1] && a.mn[2] <= b.mx[2] &&
           b.mn[2] <= a.mx[2];
}

// All (query, leaf) pairs with overlapping boxes that `keep` accepts, query
// ascending, leaf ascending, by a uniform grid over the leaves: cells of
// twice the median leaf extent, each leaf listed in every cell its box
// touches (CSR lists), each query gathering the leaves of the cells its box
// touches; leaves much larger than the typical one are tested against every
// query.  Every accepted pair is tested on the boxes themselves, so the set
// is the exact all-pairs set whatever the cell size.
template <typename Keep>
std::vector<int32_t> sweep(const std::vector<Box>& q, const std::vector<Box>& leaf, Keep keep) {
    const int nl = (int)leaf.size();
    std::vector<double> ext(nl);
    for (int i = 0; i < nl; ++i)
        ext[i] = std::max({leaf[i].mx[0] - leaf[i].mn[0], leaf[i].mx[1] - leaf[i].mn[1], leaf[i].mx[2] - leaf[i].mn[2]});
    std::vector<double> es = ext;
    std::sort(es.begin(), es.end());
    const double typical = es.empty() ? 0.0 : es[es.size() / 2];
    std::vector<int> small, big;
    for (int i = 0; i < nl; ++i) (ext[i] > 8.0 * typical + 1e-12 ? big : small).push_back(i);
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (size_t k = 0; k < small.size(); ++k)
        for (int d = 0; d < 3; ++d) {
            const Box& b = leaf[small[k]];
            lo[d] = k ? std::min(lo[d], b.mn[d]) : b.mn[d];
            hi[d] = k ? std::max(hi[d], b.mx[d]) : b.mx[d];
        }
    double h = std::max(2.0 * typical, 1e-9);
    int64_t dim[3];
    for (;;) {
        for (int d = 0; d < 3; ++d) dim[d] = std::max<int64_t>(1, (int64_t)std::floor((hi[d] - lo[d]) / h) + 1);
        if (dim[0] * dim[1] * dim[2] <= (int64_t)1 << 22) break;
        h *= 2.0;
    }
    auto cell = [&](double v, int d) {
        const int64_t c = (int64_t)std::floor((v - lo[d]) / h);
        return std::min<int64_t>(std::max<int64_t>(c, 0), dim[d] - 1);
    };
    const int64_t ncell = dim[0] * dim[1] * dim[2];
    std::vector<int64_t> start(ncell + 1, 0);
    std::vector<int32_t> items;
    for (int pass = 0; pass < 2; ++pass) {
        std::vector<int64_t> fill;
        if (pass == 1) {
            for (int64_t c = 0; c < ncell; ++c) start[c + 1] += start[c];
            items.resize(start[ncell]);
            fill.assign(start.begin(), start.end() - 1);
        }
        for (int i : small) {
            const Box& b = leaf[i];
            for (int64_t z = cell(b.mn[2], 2); z <= cell(b.mx[2], 2); ++z)
                for (int64_t y = cell(b.mn[1], 1); y <= cell(b.mx[1], 1); ++y)
                    for (int64_t x = cell(b.mn[0], 0); x <= cell(b.mx[0], 0); ++x) {
                        const int64_t c = (z * dim[1] + y) * dim[0] + x;
                        if (pass == 0) ++start[c + 1];
                        else items[fill[c]++] = i;
                    }
        }
    }
    std::vector<std::vector<int32_t>> hits(q.size());
#pragma omp parallel for schedule(dynamic, 256)
    for (long long qi = 0; qi < (long long)q.size(); ++qi) {
        const Box& Q = q[qi];
        std::vector<int32_t>& hv = hits[qi];
        bool outside = small.empty();
        for (int d = 0; d < 3; ++d) outside = outside || Q.mx[d] < lo[d] || Q.mn[d] > hi[d];
        if (!outside)
            for (int64_t z = cell(Q.mn[2], 2); z <= cell(Q.mx[2], 2); ++z)
                for (int64_t y = cell(Q.mn[1], 1); y <= cell(Q.mx[1], 1); ++y)
                    for (int64_t x = cell(Q.mn[0], 0); x <= cell(Q.mx[0], 0); ++x) {
                        const int64_t c = (z * dim[1] + y) * dim[0] + x;
                        for (int64_t k = start[c]; k < start[c + 1]; ++k) {
                            const int L = items[k];
                            if (overlap(Q, leaf[L]) && keep((int)qi, L)) hv.push_back(L);
                        }
                    }
        for (int L : big)
            if (overlap(Q, leaf[L]) && keep((int)qi, L)) hv.push_back(L);
        std::sort(hv.begin(), hv.end());
        hv.erase(std::unique(hv.begin(), hv.end()), hv.end());
    }
    std::vector<int32_t> out;
    for (size_t qi = 0; qi < q.size(); ++qi)
        for (int32_t L : hits[qi]) { out.push_back((int32_t)qi); out.push_back(L); }
    return out;
}

void candidates(const Geo& g, double infl, std::vector<int32_t>& pt, std::vector<int32_t>& ee) {
    std::vector<Box> fb(g.nf), eb(g.ne), qv(g.nv), qe(g.ne);
    for (int64_t f = 0; f < g.nf; ++f) fb[f] = box_of(g, &g.fvert[3 * f], 3, infl, g.fbody[f]);
    for (int64_t e = 0; e < g.ne; ++e) {
        eb[e] = box_of(g, &g.evert[2 * e], 2, infl, g.ebody[e]);
        qe[e] = box_of(g, &g.evert[2 * e], 2, 0.0, g.ebody[e]);
    }
    for (int64_t v = 0; v < g.nv; ++v) { const int32_t id = (int32_t)v; qv[v] = box_of(g, &id, 1, 0.0, g.vbody[v]); }
    pt = sweep(qv, fb, [&](int v, int f) { return g.vbody[v] != g.fbody[f]; });
    ee = sweep(qe, eb, [&](int a, int b) { return a < b && g.ebody[a] != g.ebody[b]; });
}

void pair_points(const Geo& g, const std::vector<int32_t>& pt, const std::vector<int32_t>& ee, size_t p, int& kind, V3* X,
                 int* side, V3* arm, int& bA, int& bB) {
    int vid[4];
    const size_t npt = pt.size() / 2;
    if (p < npt) {
        kind = ipc::kPairPT;
        const int v = pt[2 * p], f = pt[2 * p + 1];
        vid[0] = v; vid[1] = g.fvert[3 * f]; vid[2] = g.fvert[3 * f + 1]; vid[3] = g.fvert[3 * f + 2];
        bA = g.vbody[v]; bB = g.fbody[f];
        side[0] = 0; side[1] = 1; side[2] = 1; side[3] = 1;
    } else {
        kind = ipc::kPairEE;
        const size_t q = p - npt;
        const int e0 = ee[2 * q], e1 = ee[2 * q + 1];
        vid[0] = g.evert[2 * e0]; vid[1] = g.evert[2 * e0 + 1]; vid[2] = g.evert[2 * e1]; vid[3] = g.evert[2 * e1 + 1];
        bA = g.ebody[e0]; bB = g.ebody[e1];
        side[0] = 0; side[1] = 0; side[2] = 1; side[3] = 1;
    }
    for (int k = 0; k < 4; ++k) {
        X[k] = nx::ld3(&g.wv[3 * vid[k]]);
        arm[k] = X[k] - nx::ld3(&g.pos[3 * (side[k] ? bB : bA)]);
    }
}

void pair_vids(const Geo& g, const std::vector<int32_t>& pt, const std::vector<int32_t>& ee, size_t p, int* vid) {
    const size_t npt = pt.size() / 2;
    if (p < npt) {
        const int v = pt[2 * p], f = pt[2 * p + 1];
        vid[0] = v; vid[1] = g.fvert[3 * f]; vid[2] = g.fvert[3 * f + 1]; vid[3] = g.fvert[3 * f + 2];
    } else {
        const size_t q = p - npt;
        vid[0] = g.evert[2 * ee[2 * q]]; vid[1] = g.evert[2 * ee[2 * q] + 1];
        vid[2] = g.evert[2 * ee[2 * q + 1]]; vid[3] = g.evert[2 * ee[2 * q + 1] + 1];
    }
}

// the device's fixed pairwise tree (pad to a power of two, halve)
double tree_sum(std::vector<double> v) {
    size_t P = 1;
    while (P < v.size()) P <<= 1;
    v.resize(P, 0.0);
    for (size_t h = P / 2; h >= 1; h /= 2) {
        for (size_t i = 0; i < h; ++i) v[i] = v[i] + v[i + h];
        if (h == 1) break;
    }
    return v.empty() ? 0.0 : v[0];
}

// A gradient entry's or Hessian block entry's contributions (pair order),
// summed as the device's segment kernels sum them: up to 32 left to right
// from 0; more as 32 partials (partial l: contributions l, l + 32, ...,
// left to right), halved pairwise, a_l += a_{l+16}, ..., a_0 += a_1.
double seg_sum(const std::vector<double>& v) {
    if (v.size() <= 32) {
        double acc = 0.0;
        for (double t : v) acc += t;
        return acc;
    }
    double a[32] = {};
    for (size_t i = 0; i < v.size(); ++i) a[i % 32] += v[i];
    for (int off = 16; off >= 1; off /= 2)
        for (int l = 0; l < off; ++l) a[l] += a[l + off];
    return a[0];
}

// Raw 12x12 pair Hessian b'' grad grad^T + b' hess(d^2), written out densely.
void raw_hessian(const ipc::DistForm& f, const V3* X, double dhat, double kappa, double* H) {
    for (int i = 0; i < 144; ++i) H[i] = 0.0;
    const V3 r = ipc::form_r(f, X);
    const double s = nx::dot(r, r), sh = dhat * dhat;
    if (!(s < sh) || !(s > 0.0)) return;
    const double b1 = ipc::barrier_s1(s, sh, kappa), b2 = ipc::barrier_s2(s, sh, kappa);
    double gs[12];
    for (int k = 0; k < 4; ++k) { gs[3 * k] = 2.0 * f.w[k] * r.x; gs[3 * k + 1] = 2.0 * f.w[k] * r.y; gs[3 * k + 2] = 2.0 * f.w[k] * r.z; }
    V3 a[2] = {nx::v3(0, 0, 0), nx::v3(0, 0, 0)};
    for (int j = 0; j < f.nu; ++j) a[j] = f.c[0][j] * X[0] + f.c[1][j] * X[1] + f.c[2][j] * X[2] + f.c[3][j] * X[3];
    double M[2][2] = {{0, 0}, {0, 0}}, Mi[2][2] = {{0, 0}, {0, 0}};
    for (int i = 0; i < f.nu; ++i)
        for (int j = 0; j < f.nu; ++j) M[i][j] = 2.0 * nx::dot(a[i], a[j]);
    if (f.nu == 1) Mi[0][0] = 1.0 / M[0][0];
    if (f.nu == 2) {
        const double det = M[0][0] * M[1][1] - M[0][1] * M[1][0];
        Mi[0][0] = M[1][1] / det; Mi[1][1] = M[0][0] / det; Mi[0][1] = -M[0][1] / det; Mi[1][0] = -M[1][0] / det;
    }
    double G[2][12];
    for (int j = 0; j < f.nu; ++j)
        for (int k = 0; k < 4; ++k)
            for (int c = 0; c < 3; ++c) G[j][3 * k + c] = 2.0 * (f.w[k] * nx::get(a[j], c) + f.c[k][j] * nx::get(r, c));
    for (int I = 0; I < 12; ++I)
        for (int J = 0; J < 12; ++J) {
            double hs = (I % 3 == J % 3) ? 2.0 * f.w[I / 3] * f.w[J / 3] : 0.0;
            for (int p = 0; p < f.nu; ++p)
                for (int q = 0; q < f.nu; ++q) hs -= G[p][I] * Mi[p][q] * G[q][J];
            H[12 * I + J] = b2 * gs[I] * gs[J] + b1 * hs;
        }
}

}  // namespace

extern "C" {

int nxo_ipc_candidates(nxo_world* w, const double* x, const double* dx, double infl, int32_t* pt, int64_t pt_cap, int32_t* ee,
                       int64_t ee_cap, int64_t* n_pt, int64_t* n_ee) {
    const Geo g = load(w, x, dx);
    std::vector<int32_t> P, E;
    candidates(g, infl, P, E);
    *n_pt = (int64_t)P.size() / 2;
    *n_ee = (int64_t)E.size() / 2;
    if (pt) std::memcpy(pt, P.data(), sizeof(int32_t) * (size_t)std::min<int64_t>(2 * pt_cap, (int64_t)P.size()));
    if (ee) std::memcpy(ee, E.data(), sizeof(int32_t) * (size_t)std::min<int64_t>(2 * ee_cap, (int64_t)E.size()));
    return (*n_pt > pt_cap && pt) || (*n_ee > ee_cap && ee) ? NXD_CAPACITY : NXD_OK;
}

// Barrier over the candidates at x (boxes inflated by dhat): energy (fixed
// tree over all pairs, PT then EE), gradient (6N, pair order) and, when H is
// not NULL, the dense 6N x 6N PSD-projected Hessian (pair order per block).
}  // extern "C"

// nxo_ipc_barrier with, in `blocks` (when given), the body blocks the active
// pairs touch: (a, a), (a, b), (b, a), (b, b) for each, sorted by (row, col),
// the block structure of the device's BSR Hessian.
// Lagged friction of a full-IPC step (ipc::friction_pair on frozen pairs):
// `build` makes the next barrier evaluation freeze the pairs active there
// (pair order); x0 holds the step-start world vertices, taken at the first
// build.  The last evaluation's friction energy is in `energy`.
struct IpcFricCtx {
    double mu = 0.0, eps = 1e-8;
    bool build = true;
    bool only = false;   // gradient and Hessian of the friction alone
    std::vector<double> x0;
    struct Pair { int vid[4], body[2], kind; ipc::FricLag L; };
    std::vector<Pair> set;
    double energy = 0.0;
};
IpcFricCtx* ipc_fric_new(double mu, double eps) {
    auto* f = new IpcFricCtx();
    f->mu = mu; f->eps = eps;
    return f;
}
void ipc_fric_free(IpcFricCtx* f) { delete f; }
void ipc_fric_rebuild(IpcFricCtx* f) { f->build = true; }
int64_t ipc_fric_count(const IpcFricCtx* f) { return (int64_t)f->set.size(); }
double ipc_fric_energy(const IpcFricCtx* f) { return f->energy; }

int ipc_barrier_cpu(nxo_world* w, const double* x, double dhat, double kappa, double* energy, double* grad, double* H,
                    std::vector<std::pair<int, int>>* blocks, int64_t* n_pairs, int64_t* n_active, IpcFricCtx* fr);

extern "C" {

int nxo_ipc_barrier(nxo_world* w, const double* x, double dhat, double kappa, double* energy, double* grad, double* H,
                    int64_t* n_pairs, int64_t* n_active) {
    return ipc_barrier_cpu(w, x, dhat, kappa, energy, grad, H, nullptr, n_pairs, n_active, nullptr);
}

// Friction alone, for checking its derivatives: the pairs active at x_lag
// frozen there (x0 = the world vertices at x_lag), the friction energy,
// gradient (6N) and Gauss-Newton Hessian (dense 6N x 6N, or NULL) at x.
int nxo_ipc_friction(nxo_world* w, const double* x_lag, const double* x, double dhat, double kappa, double mu, double eps,
                     double* energy, double* grad, double* H, int64_t* n_friction) {
    IpcFricCtx fr;
    fr.mu = mu; fr.eps = eps; fr.only = true;
    const int N6 = 6 * nxo_body_count(w);
    std::vector<double> g(N6);
    double e = 0.0;
    ipc_barrier_cpu(w, x_lag, dhat, kappa, &e, g.data(), nullptr, nullptr, nullptr, nullptr, &fr);
    ipc_barrier_cpu(w, x, dhat, kappa, &e, grad, H, nullptr, nullptr, nullptr, &fr);
    *energy = fr.energy;
    if (n_friction) *n_friction = (int64_t)fr.set.size();
    return NXD_OK;
}

}  // extern "C"

int ipc_barrier_cpu(nxo_world* w, const double* x, double dhat, double kappa, double* energy, double* grad, double* H,
                    std::vector<std::pair<int, int>>* blocks, int64_t* n_pairs, int64_t* n_active, IpcFricCtx* fr) {
    const Geo g = load(w, x, nullptr);
    std::vector<int32_t> P, E;
    candidates(g, dhat, P, E);
    const size_t n = P.size() / 2 + E.size() / 2;
    const int N6 = 6 * g.N;
    std::vector<double> e(n);
    if (grad) std::fill(grad, grad + N6, 0.0);
    if (H) std::fill(H, H + (size_t)N6 * N6, 0.0);
    // per active pair (pair order): its bodies, chained gradient (12) and,
    // with H, its four 6x6 blocks (r, c) = (0,0), (0,1), (1,0), (1,1)
    std::vector<int> ab;
    std::vector<double> ag, ah;
    for (size_t p = 0; p < n; ++p) {
        int kind, side[4], bA, bB;
        V3 X[4], arm[4];
        pair_points(g, P, E, p, kind, X, side, arm, bA, bB);
        const ipc::DistForm f = ipc::classify(kind, X);
        const ipc::PairEval ev = ipc::pair_barrier(f, X, dhat, kappa);
        e[p] = ev.e;
        if (!(ev.d2 < dhat * dhat)) continue;
        if (blocks) {
            blocks->push_back({bA, bA}); blocks->push_back({bA, bB});
            blocks->push_back({bB, bA}); blocks->push_back({bB, bB});
        }
        ab.push_back(bA); ab.push_back(bB);
        double g12[12];
        const V3 thA = nx::ld3(&g.theta[3 * bA]), thB = nx::ld3(&g.theta[3 * bB]);
        ipc::chain12_exact(ev.grad, side, arm, thA, thB, g12);
        ag.insert(ag.end(), g12, g12 + 12);
        if (!H) continue;
        double z[5][12];
        for (int k = 0; k < ev.n_terms; ++k) ipc::chain12_exact(ev.y[k], side, arm, thA, thB, z[k]);
        for (int r = 0; r < 2; ++r)
            for (int c = 0; c < 2; ++c)
                for (int i = 0; i < 6; ++i)
                    for (int j = 0; j < 6; ++j) {
                        double blk = 0.0;
                        for (int k = 0; k < ev.n_terms; ++k) blk += (ev.lam[k] * z[k][6 * r + i]) * z[k][6 * c + j];
                        ah.push_back(blk);
                    }
    }
    const size_t nbar = ab.size() / 2;
    if (fr && fr->only) {
        ab.clear(); ag.clear(); ah.clear();
        if (blocks) blocks->clear();
    }
    if (fr && fr->build) {
        // freeze the active pairs here (pair order)
        fr->build = false;
        if (fr->x0.empty()) fr->x0 = g.wv;
        fr->set.clear();
        for (size_t p = 0; p < n; ++p) {
            int kind, side[4], bA, bB;
            V3 X[4], arm[4];
            pair_points(g, P, E, p, kind, X, side, arm, bA, bB);
            const ipc::DistForm f = ipc::classify(kind, X);
            IpcFricCtx::Pair fp;
            if (!ipc::friction_lag(f, X, dhat, kappa, fp.L)) continue;
            pair_vids(g, P, E, p, fp.vid);
            fp.body[0] = bA; fp.body[1] = bB; fp.kind = kind;
            fr->set.push_back(fp);
        }
    }
    if (fr) {
        // the frozen pairs after the active barrier pairs, energies in their own tree
        std::vector<double> ef(fr->set.size());
        for (size_t q = 0; q < fr->set.size(); ++q) {
            const IpcFricCtx::Pair& fp = fr->set[q];
            const int side[4] = {0, fp.kind == ipc::kPairPT ? 1 : 0, 1, 1};
            V3 X[4], X0[4], arm[4];
            for (int k = 0; k < 4; ++k) {
                X[k] = nx::ld3(&g.wv[3 * fp.vid[k]]);
                X0[k] = nx::ld3(&fr->x0[3 * fp.vid[k]]);
                arm[k] = X[k] - nx::ld3(&g.pos[3 * fp.body[side[k]]]);
            }
            const ipc::FricEval ev = ipc::friction_pair(fp.L, X, X0, fr->mu, fr->eps);
            ef[q] = ev.e;
            ab.push_back(fp.body[0]); ab.push_back(fp.body[1]);
            double g12[12];
            const V3 thA = nx::ld3(&g.theta[3 * fp.body[0]]), thB = nx::ld3(&g.theta[3 * fp.body[1]]);
            ipc::chain12_exact(ev.grad, side, arm, thA, thB, g12);
            ag.insert(ag.end(), g12, g12 + 12);
            if (!H) continue;
            double z[2][12];
            for (int k = 0; k < 2; ++k) ipc::chain12_exact(ev.y[k], side, arm, thA, thB, z[k]);
            for (int r = 0; r < 2; ++r)
                for (int c = 0; c < 2; ++c)
                    for (int i = 0; i < 6; ++i)
                        for (int j = 0; j < 6; ++j) {
                            double blk = 0.0;
                            for (int k = 0; k < 2; ++k) blk += (ev.lam[k] * z[k][6 * r + i]) * z[k][6 * c + j];
                            ah.push_back(blk);
                        }
            if (blocks) {
                blocks->push_back({fp.body[0], fp.body[0]}); blocks->push_back({fp.body[0], fp.body[1]});
                blocks->push_back({fp.body[1], fp.body[0]}); blocks->push_back({fp.body[1], fp.body[1]});
            }
        }
        fr->energy = tree_sum(ef);
    }
    const size_t na = ab.size() / 2;
    // each gradient entry / block entry: its contributions in pair order,
    // summed as the device sums a segment (seg_sum)
    std::vector<double> vals;
    if (grad) {
        std::vector<std::vector<std::pair<int, int>>> seg(g.N);   // (active pair, side)
        for (size_t a = 0; a < na; ++a)
            for (int sd = 0; sd < 2; ++sd) seg[ab[2 * a + sd]].push_back({(int)a, sd});
        for (int b = 0; b < g.N; ++b)
            for (int d = 0; seg[b].size() && d < 6; ++d) {
                vals.clear();
                for (const auto& t : seg[b]) vals.push_back(ag[12 * (size_t)t.first + 6 * t.second + d]);
                grad[6 * b + d] = seg_sum(vals);
            }
    }
    if (H) {
        std::map<std::pair<int, int>, std::vector<std::pair<int, int>>> seg;   // (row, col body) -> (active pair, block)
        for (size_t a = 0; a < na; ++a)
            for (int r = 0; r < 2; ++r)
                for (int c = 0; c < 2; ++c) seg[{ab[2 * a + r], ab[2 * a + c]}].push_back({(int)a, 2 * r + c});
        for (const auto& kv : seg)
            for (int i = 0; i < 6; ++i)
                for (int j = 0; j < 6; ++j) {
                    vals.clear();
                    for (const auto& t : kv.second) vals.push_back(ah[144 * (size_t)t.first + 36 * t.second + 6 * i + j]);
                    H[(size_t)(6 * kv.first.first + i) * N6 + 6 * kv.first.second + j] = seg_sum(vals);
                }
    }
    if (energy) *energy = tree_sum(e);
    if (n_pairs) *n_pairs = (int64_t)n;
    if (n_active) *n_active = (int64_t)nbar;
    if (blocks) {
        std::sort(blocks->begin(), blocks->end());
        blocks->erase(std::unique(blocks->begin(), blocks->end()), blocks->end());
    }
    return NXD_OK;
}

extern "C" {

// Largest step fraction in [0, 1] along x -> x + dx that additive CCD allows
// (eta: kept fraction of each pair's initial distance), over the pairs whose
// swept boxes overlap.
double nxo_ipc_max_step(nxo_world* w, const double* x, const double* dx, double eta, int64_t* n_pairs) {
    const Geo g = load(w, x, dx);
    std::vector<int32_t> P, E;
    candidates(g, 0.0, P, E);
    const size_t n = P.size() / 2 + E.size() / 2;
    if (n_pairs) *n_pairs = (int64_t)n;
    double t = 1.0;
    for (size_t p = 0; p < n; ++p) {
        int kind, side[4], bA, bB;
        V3 X[4], arm[4];
        pair_points(g, P, E, p, kind, X, side, arm, bA, bB);
        int vid[4];
        pair_vids(g, P, E, p, vid);
        // along the rigid arcs x + t dx (ipc::ArcMotion)
        ipc::ArcMotion m;
        m.kind = kind;
        const int b[2] = {bA, bB};
        for (int sd = 0; sd < 2; ++sd) {
            m.b[sd].p = nx::ld3(&g.x[6 * b[sd]]);
            m.b[sd].th = nx::ld3(&g.x[6 * b[sd] + 3]);
            m.b[sd].dp = nx::ld3(&g.dx[6 * b[sd]]);
            m.b[sd].dth = nx::ld3(&g.dx[6 * b[sd] + 3]);
            m.b[sd].q0 = nx::ldq(&g.quat[4 * b[sd]]);
        }
        for (int k = 0; k < 4; ++k) { m.side[k] = side[k]; m.v[k] = nx::ld3(&g.vloc[3 * vid[k]]); }
        t = nx::dmin(t, ipc::accd_toi_motion(kind, m, 1.0, eta, 1000, nullptr));
    }
    return t;
}

// One pair (X12 = four points): d^2, type, energy, gradient (12), the
// subspace PSD Hessian (144), the raw Hessian (144) and its PSD projection
// by a full 12x12 Jacobi decomposition (144).  Any output may be NULL.
int nxo_ipc_pair(int32_t kind, const double* X12, double dhat, double kappa, double* d2, int32_t* type, double* e, double* g12,
                 double* H_sub, double* H_raw, double* H_full) {
    V3 X[4];
    for (int k = 0; k < 4; ++k) X[k] = nx::ld3(X12 + 3 * k);
    const ipc::DistForm f = ipc::classify(kind, X);
    const ipc::PairEval ev = ipc::pair_barrier(f, X, dhat, kappa);
    if (d2) *d2 = ev.d2;
    if (type) *type = f.type;
    if (e) *e = ev.e;
    if (g12)
        for (int k = 0; k < 4; ++k) nx::st3(g12 + 3 * k, ev.grad.v[k]);
    if (H_sub) {
        for (int i = 0; i < 144; ++i) H_sub[i] = 0.0;
        for (int k = 0; k < ev.n_terms; ++k)
            for (int I = 0; I < 12; ++I)
                for (int J = 0; J < 12; ++J)
                    H_sub[12 * I + J] += ev.lam[k] * nx::get(ev.y[k].v[I / 3], I % 3) * nx::get(ev.y[k].v[J / 3], J % 3);
    }
    double R[144];
    raw_hessian(f, X, dhat, kappa, R);
    if (H_raw) std::memcpy(H_raw, R, sizeof(R));
    if (H_full) {
        double A[12][12], V[12][12];
        for (int i = 0; i < 12; ++i)
            for (int j = 0; j < 12; ++j) A[i][j] = 0.5 * (R[12 * i + j] + R[12 * j + i]);
        ipc::jacobi_eigen<12>(A, V, 12);
        for (int i = 0; i < 12; ++i)
            for (int j = 0; j < 12; ++j) {
                double h = 0.0;
                for (int k = 0; k < 12; ++k)
                    if (A[k][k] > 0.0) h += A[k][k] * V[i][k] * V[j][k];
                H_full[12 * i + j] = h;
            }
    }
    return NXD_OK;
}

double nxo_ipc_accd(int32_t kind, const double* X12, const double* D12, double t_max, double eta, int32_t max_iter,
                    int32_t* iters) {
    V3 X[4], D[4];
    for (int k = 0; k < 4; ++k) { X[k] = nx::ld3(X12 + 3 * k); D[k] = nx::ld3(D12 + 3 * k); }
    int it = 0;
    const double t = ipc::accd_toi(kind, X, D, t_max, eta, max_iter, &it);
    if (iters) *iters = it;
    return t;
}

// One frozen pair's friction point forces and their derivatives with respect
// to the points (H) and to the lag points (Hs), ipc::friction_derivs; the
// distance type of the lag points in *type.
void nxo_ipc_friction_derivs(int32_t kind, const double* X12, const double* Xs12, double dhat, double kappa, double mu,
                             double eps, double* g12, double* H, double* Hs, int32_t* type) {
    V3 X[4], Xs[4];
    for (int k = 0; k < 4; ++k) { X[k] = nx::ld3(X12 + 3 * k); Xs[k] = nx::ld3(Xs12 + 3 * k); }
    const ipc::DistForm fs = ipc::classify(kind, Xs);
    if (type) *type = fs.type;
    ipc::friction_derivs(fs, X, Xs, dhat, kappa, mu, eps, g12, H, Hs);
}

double nxo_ipc_dist2(int32_t kind, const double* X12) {
    V3 X[4];
    for (int k = 0; k < 4; ++k) X[k] = nx::ld3(X12 + 3 * k);
    return ipc::dist2(kind, X);
}

}  // extern "C"
