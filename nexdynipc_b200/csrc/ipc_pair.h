// ipc_pair.h — per-pair arithmetic of the primitive-level contact model
// (full IPC, "Mode I"): distance-type classification, squared distance with
// its gradient and Hessian, the log barrier on squared distance, the PSD
// projection of the pair Hessian, the chain to rigid-body DOFs, and additive
// CCD.  Shared by the sm_100a kernels and the CPU oracle (compiled without
// FMA contraction on both sides).  The reference has no such model; the
// formulas follow the published methods:
//   Li et al. 2020, "Incremental Potential Contact" (barrier on squared
//     distance, distance types, PSD-projected Hessians);
//   Ericson 2005, "Real-Time Collision Detection" 5.1.9 (clamped closest
//     points of two segments), 5.1.5 (closest point on a triangle by regions);
//   Li et al. 2021, "Codimensional Incremental Potential Contact" (additive
//     CCD: conservative advancement with a Lipschitz bound on the distance).
//
// Every pair has four points X[0..3]: point-triangle (p, t0, t1, t2),
// edge-edge (a0, a1, b0, b1).  A classified pair is a DistForm: the squared
// distance is |r|^2 with r = sum_k w_k X_k, the weights affine in nu <= 2
// parameters u whose optimum the type fixes (c[k][j] = dw_k / du_j).  With
// g(x, u) = |r|^2 and f(x) = min_u g:
//   grad_k f = 2 w_k r,
//   hess f   = g_xx - g_xu g_uu^-1 g_ux,  g_xx = 2 (w w^T) (x) I3,
//   g_uu = 2 A^T A (A = [a_j], a_j = sum_k c_kj X_k),
//   g_{x_k u_j} = 2 (w_k a_j + c_kj r).
// The Hessian's range lies in span{w (x) e_1..3, c_1 (x) r, c_2 (x) r}, so
// the barrier Hessian b'' grad grad^T + b' hess is projected to PSD exactly
// by an eigen-decomposition in that <= 5-dimensional basis.
#pragma once

#include "nx_math.cuh"

namespace nx {
namespace ipc {

enum { kPairPT = 0, kPairEE = 1 };

// Type codes.  PT: 0..2 point-vertex (t0, t1, t2), 3..5 point-edge (t0t1,
// t1t2, t2t0), 6 point-interior.  EE: 0..3 vertex-vertex (a0b0, a0b1, a1b0,
// a1b1), 4..5 a-edge vs b0 / b1, 6..7 b-edge vs a0 / a1, 8 interior.
struct DistForm {
    double w[4];
    double c[4][2];
    int nu;
    int type;
};

struct V12 { V3 v[4]; };

NX_HD DistForm form_zero() {
    DistForm f;
    for (int k = 0; k < 4; ++k) { f.w[k] = 0.0; f.c[k][0] = 0.0; f.c[k][1] = 0.0; }
    f.nu = 0; f.type = 0;
    return f;
}
NX_HD double clamp01(double v) { return v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v); }

// Point p = X[0] against the segment X[i] X[j]: clamped parameter and d^2.
NX_HD double point_segment(const V3* X, int i, int j, double& t) {
    const V3 e = X[j] - X[i];
    const double ee = dot(e, e);
    t = ee > 0.0 ? clamp01(dot(X[0] - X[i], e) / ee) : 0.0;
    const V3 r = X[0] - X[i] - t * e;
    return dot(r, r);
}

// Point-triangle classification (p, t0, t1, t2).
NX_HD DistForm classify_pt(const V3* X) {
    DistForm f = form_zero();
    const V3 e1 = X[2] - X[1], e2 = X[3] - X[1], q = X[0] - X[1];
    const double a = dot(e1, e1), b = dot(e1, e2), c = dot(e2, e2), d = dot(e1, q), e = dot(e2, q);
    const double det = a * c - b * b;
    if (det > 1e-14 * a * c) {
        const double b1 = (c * d - b * e) / det, b2 = (a * e - b * d) / det;
        if (b1 >= 0.0 && b2 >= 0.0 && b1 + b2 <= 1.0) {
            f.w[0] = 1.0; f.w[1] = -(1.0 - b1 - b2); f.w[2] = -b1; f.w[3] = -b2;
            f.c[1][0] = 1.0; f.c[1][1] = 1.0; f.c[2][0] = -1.0; f.c[3][1] = -1.0;
            f.nu = 2; f.type = 6;
            return f;
        }
    }
    // boundary: the nearest of the three edges (first minimum in order)
    const int ei[3] = {1, 2, 3}, ej[3] = {2, 3, 1};
    double best = 0.0, bt = 0.0;
    int be = -1;
    for (int k = 0; k < 3; ++k) {
        double t;
        const double d2 = point_segment(X, ei[k], ej[k], t);
        if (be < 0 || d2 < best) { best = d2; bt = t; be = k; }
    }
    const int i = ei[be], j = ej[be];
    f.w[0] = 1.0;
    if (bt > 0.0 && bt < 1.0) {
        f.w[i] = -(1.0 - bt); f.w[j] = -bt;
        f.c[i][0] = 1.0; f.c[j][0] = -1.0;
        f.nu = 1; f.type = 3 + be;
    } else {
        const int v = bt <= 0.0 ? i : j;
        f.w[v] = -1.0;
        f.nu = 0; f.type = v - 1;
    }
    return f;
}

// Edge-edge classification (a0, a1, b0, b1), clamped closest points.
// Nearly parallel edges (A E - B^2 <= 1e-10 A E) take s = 0, so they never
// classify as interior.
NX_HD DistForm classify_ee(const V3* X) {
    DistForm f = form_zero();
    const V3 d1 = X[1] - X[0], d2 = X[3] - X[2], r = X[0] - X[2];
    const double A = dot(d1, d1), E = dot(d2, d2), F = dot(d2, r);
    double s = 0.0, t = 0.0;
    if (A <= 1e-30 && E <= 1e-30) {
        s = 0.0; t = 0.0;
    } else if (A <= 1e-30) {
        s = 0.0; t = clamp01(F / E);
    } else {
        const double C = dot(d1, r);
        if (E <= 1e-30) {
            t = 0.0; s = clamp01(-C / A);
        } else {
            const double B = dot(d1, d2);
            const double den = A * E - B * B;
            s = den > 1e-10 * A * E ? clamp01((B * F - C * E) / den) : 0.0;
            t = (B * s + F) / E;
            if (t < 0.0) { t = 0.0; s = clamp01(-C / A); }
            else if (t > 1.0) { t = 1.0; s = clamp01((B - C) / A); }
        }
    }
    const bool si = s > 0.0 && s < 1.0, ti = t > 0.0 && t < 1.0;
    if (si && ti) {
        f.w[0] = 1.0 - s; f.w[1] = s; f.w[2] = -(1.0 - t); f.w[3] = -t;
        f.c[0][0] = -1.0; f.c[1][0] = 1.0; f.c[2][1] = 1.0; f.c[3][1] = -1.0;
        f.nu = 2; f.type = 8;
    } else if (si) {
        const int pb = t <= 0.0 ? 2 : 3;
        f.w[0] = 1.0 - s; f.w[1] = s; f.w[pb] = -1.0;
        f.c[0][0] = -1.0; f.c[1][0] = 1.0;
        f.nu = 1; f.type = 4 + (pb - 2);
    } else if (ti) {
        const int pa = s <= 0.0 ? 0 : 1;
        f.w[pa] = 1.0; f.w[2] = -(1.0 - t); f.w[3] = -t;
        f.c[2][0] = 1.0; f.c[3][0] = -1.0;
        f.nu = 1; f.type = 6 + pa;
    } else {
        const int pa = s <= 0.0 ? 0 : 1, pb = t <= 0.0 ? 2 : 3;
        f.w[pa] = 1.0; f.w[pb] = -1.0;
        f.nu = 0; f.type = 2 * pa + (pb - 2);
    }
    return f;
}

NX_HD DistForm classify(int kind, const V3* X) { return kind == kPairPT ? classify_pt(X) : classify_ee(X); }

NX_HD V3 form_r(const DistForm& f, const V3* X) {
    return f.w[0] * X[0] + f.w[1] * X[1] + f.w[2] * X[2] + f.w[3] * X[3];
}
NX_HD double dist2(int kind, const V3* X) {
    const DistForm f = classify(kind, X);
    const V3 r = form_r(f, X);
    return dot(r, r);
}

// Log barrier on squared distance s with support s < sh = dhat^2:
// b(s) = -kappa (s - sh)^2 ln(s / sh), and its first two derivatives in s.
NX_HD double barrier_s(double s, double sh, double kappa) {
    if (!(s < sh)) return 0.0;
    if (!(s > 0.0)) return INFINITY;
    const double q = s - sh;
    return -kappa * q * q * nxm::log(s / sh);
}
NX_HD double barrier_s1(double s, double sh, double kappa) {
    if (!(s < sh) || !(s > 0.0)) return 0.0;
    const double q = s - sh;
    return -kappa * (2.0 * q * nxm::log(s / sh) + q * q / s);
}
NX_HD double barrier_s2(double s, double sh, double kappa) {
    if (!(s < sh) || !(s > 0.0)) return 0.0;
    const double q = s - sh;
    return -kappa * (2.0 * nxm::log(s / sh) + 4.0 * q / s - (q * q) / (s * s));
}

// Cyclic Jacobi eigen-decomposition of a symmetric m x m matrix (m <= 5),
// in place: on return A holds the eigenvalues on its diagonal and V the
// eigenvectors (columns).  At most 16 sweeps.  Loops run to the fixed bound
// M with m as a guard, so every index is a compile-time constant once
// unrolled (the matrices can stay in registers); the operations and their
// order are those of loops to m.
template <int M>
NX_HD void jacobi_eigen(double (&A)[M][M], double (&V)[M][M], int m) {
NX_UNROLL
    for (int i = 0; i < M; ++i)
NX_UNROLL
        for (int j = 0; j < M; ++j) V[i][j] = i == j ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 16; ++sweep) {
        double off = 0.0, tot = 0.0;
NX_UNROLL
        for (int i = 0; i < M; ++i)
NX_UNROLL
            for (int j = 0; j < M; ++j) {
                if (i >= m || j >= m) continue;
                tot += A[i][j] * A[i][j];
                if (i != j) off += A[i][j] * A[i][j];
            }
        if (!(off > 1e-30 * tot)) break;
NX_UNROLL
        for (int p = 0; p < M - 1; ++p)
NX_UNROLL
            for (int q = p + 1; q < M; ++q) {
                if (q >= m) continue;
                const double apq = A[p][q];
                if (apq == 0.0) continue;
                const double theta = (A[q][q] - A[p][p]) / (2.0 * apq);
                const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
NX_UNROLL
                for (int k = 0; k < M; ++k) {
                    if (k >= m) continue;
                    const double akp = A[k][p], akq = A[k][q];
                    A[k][p] = c * akp - s * akq;
                    A[k][q] = s * akp + c * akq;
                }
NX_UNROLL
                for (int k = 0; k < M; ++k) {
                    if (k >= m) continue;
                    const double apk = A[p][k], aqk = A[q][k];
                    A[p][k] = c * apk - s * aqk;
                    A[q][k] = s * apk + c * aqk;
                }
NX_UNROLL
                for (int k = 0; k < M; ++k) {
                    if (k >= m) continue;
                    const double vkp = V[k][p], vkq = V[k][q];
                    V[k][p] = c * vkp - s * vkq;
                    V[k][q] = s * vkp + c * vkq;
                }
            }
    }
}

// 12-vectors as four V3 blocks.
NX_HD double dot12(const V12& a, const V12& b) {
    return (dot(a.v[0], b.v[0]) + dot(a.v[1], b.v[1])) + (dot(a.v[2], b.v[2]) + dot(a.v[3], b.v[3]));
}
NX_HD void axpy12(double s, const V12& x, V12& y) {
    for (int k = 0; k < 4; ++k) y.v[k] = y.v[k] + s * x.v[k];
}
NX_HD V12 scale12(double s, const V12& x) {
    V12 y;
    for (int k = 0; k < 4; ++k) y.v[k] = s * x.v[k];
    return y;
}
NX_HD V12 outer_wv(const double* w, V3 v) {   // w (x) v
    V12 y;
    for (int k = 0; k < 4; ++k) y.v[k] = w[k] * v;
    return y;
}

// Barrier of one classified pair.  Outputs: e = b(d^2); grad (12) =
// b' grad d^2; the PSD part of the Hessian as sum_k lam[k] y_k y_k^T with
// at most 5 terms (n_terms).  Returns d^2.
struct PairEval {
    double d2, e;
    V12 grad;
    int n_terms;
    double lam[5];
    V12 y[5];
};

NX_HD PairEval pair_barrier(const DistForm& f, const V3* X, double dhat, double kappa) {
    PairEval o;
    const V3 r = form_r(f, X);
    const double s = dot(r, r), sh = dhat * dhat;
    o.d2 = s;
    o.e = barrier_s(s, sh, kappa);
    o.n_terms = 0;
    for (int k = 0; k < 4; ++k) o.grad.v[k] = v3(0, 0, 0);
    if (!(s < sh) || !(s > 0.0)) return o;
    const double b1 = barrier_s1(s, sh, kappa), b2 = barrier_s2(s, sh, kappa);
    const V12 gs = outer_wv(f.w, 2.0 * r);          // grad d^2
    o.grad = scale12(b1, gs);
    // a_j, g_uu = 2 A^T A, its inverse
    V3 a[2] = {v3(0, 0, 0), v3(0, 0, 0)};
    for (int j = 0; j < f.nu; ++j)
        a[j] = f.c[0][j] * X[0] + f.c[1][j] * X[1] + f.c[2][j] * X[2] + f.c[3][j] * X[3];
    double Minv[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
    if (f.nu == 1) {
        Minv[0][0] = 1.0 / (2.0 * dot(a[0], a[0]));
    } else if (f.nu == 2) {
        const double m00 = 2.0 * dot(a[0], a[0]), m01 = 2.0 * dot(a[0], a[1]), m11 = 2.0 * dot(a[1], a[1]);
        const double det = m00 * m11 - m01 * m01;
        Minv[0][0] = m11 / det; Minv[0][1] = -m01 / det; Minv[1][0] = -m01 / det; Minv[1][1] = m00 / det;
    }
    // G_j = 2 (w (x) a_j + c_j (x) r)
    V12 G[2];
    for (int j = 0; j < f.nu; ++j) {
        const double cj[4] = {f.c[0][j], f.c[1][j], f.c[2][j], f.c[3][j]};
        G[j] = outer_wv(f.w, 2.0 * a[j]);
        axpy12(1.0, outer_wv(cj, 2.0 * r), G[j]);
    }
    // orthonormal basis: w (x) e_a / |w| (a = x, y, z), then the c_j (x) r
    // directions orthogonalised against it (twice, modified Gram-Schmidt)
    const double wn = sqrt((f.w[0] * f.w[0] + f.w[1] * f.w[1]) + (f.w[2] * f.w[2] + f.w[3] * f.w[3]));
    // (loops below run to fixed bounds with the runtime sizes as guards, so
    // that every array index is a compile-time constant once unrolled; the
    // operations and their order are those of loops to m and nu)
    V12 B[5];
    const V3 ex = v3(1, 0, 0), ey = v3(0, 1, 0), ez = v3(0, 0, 1);
    B[0] = outer_wv(f.w, (1.0 / wn) * ex);
    B[1] = outer_wv(f.w, (1.0 / wn) * ey);
    B[2] = outer_wv(f.w, (1.0 / wn) * ez);
    int m = 3;
NX_UNROLL
    for (int j = 0; j < 2; ++j) {
        if (j >= f.nu) continue;
        const double cj[4] = {f.c[0][j], f.c[1][j], f.c[2][j], f.c[3][j]};
        V12 v = outer_wv(cj, r);
        const double n0 = sqrt(dot12(v, v));
NX_UNROLL
        for (int pass = 0; pass < 2; ++pass)
NX_UNROLL
            for (int k = 0; k < 4; ++k)
                if (k < m) axpy12(-dot12(B[k], v), B[k], v);
        const double n1 = sqrt(dot12(v, v));
        if (n1 > 1e-9 * n0 && n1 > 0.0) {
            const V12 u = scale12(1.0 / n1, v);
            if (m == 3) B[3] = u;
            else B[4] = u;
            ++m;
        }
    }
    // coordinates of grad d^2 and G_j in the basis; the basis image of
    // 2 (w w^T) (x) I3 is 2 |w|^2 on the first three coordinates
    double gam[5], Gam[2][5];
NX_UNROLL
    for (int k = 0; k < 5; ++k) {
        if (k >= m) continue;
        gam[k] = dot12(B[k], gs);
NX_UNROLL
        for (int j = 0; j < 2; ++j)
            if (j < f.nu) Gam[j][k] = dot12(B[k], G[j]);
    }
    double S[5][5], V[5][5];
NX_UNROLL
    for (int i = 0; i < 5; ++i)
NX_UNROLL
        for (int j = 0; j < 5; ++j) S[i][j] = 0.0;
NX_UNROLL
    for (int i = 0; i < 5; ++i)
NX_UNROLL
        for (int j = 0; j < 5; ++j) {
            if (i >= m || j >= m) continue;
            double hs = (i == j && i < 3) ? 2.0 * wn * wn : 0.0;
NX_UNROLL
            for (int p = 0; p < 2; ++p)
NX_UNROLL
                for (int q = 0; q < 2; ++q)
                    if (p < f.nu && q < f.nu) hs -= Gam[p][i] * Minv[p][q] * Gam[q][j];
            S[i][j] = b2 * gam[i] * gam[j] + b1 * hs;
        }
NX_UNROLL
    for (int i = 0; i < 5; ++i)
NX_UNROLL
        for (int j = 0; j < i; ++j) {   // exact symmetry before the rotations
            if (i >= m) continue;
            const double avg = 0.5 * (S[i][j] + S[j][i]);
            S[i][j] = avg; S[j][i] = avg;
        }
    jacobi_eigen<5>(S, V, m);
    int n = 0;
NX_UNROLL
    for (int k = 0; k < 5; ++k) {
        if (k >= m) continue;
        const double lam = S[k][k];
        if (!(lam > 0.0)) continue;
        V12 y = scale12(V[0][k], B[0]);
NX_UNROLL
        for (int i = 1; i < 5; ++i)
            if (i < m) axpy12(V[i][k], B[i], y);
        o.lam[n] = lam;
        o.y[n] = y;
        ++n;
    }
    o.n_terms = n;
    return o;
}

// Exact (unprojected) barrier of one classified pair in point space, for the
// step adjoint, which differentiates the gradient itself: g12 = b' grad d^2
// and the 12 x 12 row-major Hessian H = b'' grad grad^T + b' hess d^2 with
// hess d^2 = g_xx - sum_pq G_p (g_uu^-1)_pq G_q^T (the envelope formula of
// the header comment).  Zero outside the barrier's support.  Returns d^2.
NX_HD double pair_barrier_exact(const DistForm& f, const V3* X, double dhat, double kappa, double* g12, double* H) {
    const V3 r = form_r(f, X);
    const double s = dot(r, r), sh = dhat * dhat;
    for (int i = 0; i < 12; ++i) g12[i] = 0.0;
    for (int i = 0; i < 144; ++i) H[i] = 0.0;
    if (!(s < sh) || !(s > 0.0)) return s;
    const double b1 = barrier_s1(s, sh, kappa), b2 = barrier_s2(s, sh, kappa);
    double gs[12];
    for (int k = 0; k < 4; ++k) {
        gs[3 * k] = f.w[k] * (2.0 * r.x); gs[3 * k + 1] = f.w[k] * (2.0 * r.y); gs[3 * k + 2] = f.w[k] * (2.0 * r.z);
    }
    for (int i = 0; i < 12; ++i) g12[i] = b1 * gs[i];
    V3 a[2] = {v3(0, 0, 0), v3(0, 0, 0)};
    for (int j = 0; j < f.nu; ++j)
        a[j] = f.c[0][j] * X[0] + f.c[1][j] * X[1] + f.c[2][j] * X[2] + f.c[3][j] * X[3];
    double Minv[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
    if (f.nu == 1) {
        Minv[0][0] = 1.0 / (2.0 * dot(a[0], a[0]));
    } else if (f.nu == 2) {
        const double m00 = 2.0 * dot(a[0], a[0]), m01 = 2.0 * dot(a[0], a[1]), m11 = 2.0 * dot(a[1], a[1]);
        const double det = m00 * m11 - m01 * m01;
        Minv[0][0] = m11 / det; Minv[0][1] = -m01 / det; Minv[1][0] = -m01 / det; Minv[1][1] = m00 / det;
    }
    double G[2][12];
    for (int j = 0; j < 2; ++j)
        for (int k = 0; k < 4; ++k) {
            const V3 v = j < f.nu ? f.w[k] * (2.0 * a[j]) + f.c[k][j] * (2.0 * r) : v3(0, 0, 0);
            G[j][3 * k] = v.x; G[j][3 * k + 1] = v.y; G[j][3 * k + 2] = v.z;
        }
    for (int i = 0; i < 12; ++i)
        for (int j = 0; j < 12; ++j) {
            double hs = (i % 3 == j % 3) ? 2.0 * (f.w[i / 3] * f.w[j / 3]) : 0.0;
            for (int p = 0; p < f.nu; ++p)
                for (int q = 0; q < f.nu; ++q) hs -= G[p][i] * Minv[p][q] * G[q][j];
            H[12 * i + j] = b2 * gs[i] * gs[j] + b1 * hs;
        }
    return s;
}

// ---------------------------------------------------------------------------
// Lagged friction on a primitive pair: the reference's smoothed friction
// potential (FrictionPotential::value / gradient / hessian, Friction.cpp:5-61)
//   D = mu lam (sqrt(|u|^2 + eps^2) - eps),
// u the tangential displacement, here of the pair's closest points, with
// the normal force, the normal and the closest-point weights frozen at a lag
// state (the reference re-detects contacts and recomputes normal forces at
// each outer iterate, IPCSolver.cpp:1112-1130):
//   u = P sum_k w_k (X_k - X0_k),  P = I - n n^T,
// X0 the points at the step start, w_k the DistForm weights (r = sum w_k X_k
// runs from the closest point on B to the one on A), n = r / |r| and
// lam = -db/dd = -2 d b'(d^2) at the lag state.  In the points the
// Hessian mu lam / s (P - u u^T / s^2), s = sqrt(|u|^2 + eps^2), is PSD:
// mu lam eps^2 / s^3 along u, mu lam / s across it in the tangent plane, 0
// along n, i.e. two rank-one terms lam_m (w (x) t_m)(w (x) t_m)^T.  Below
// |u| = 1e-12 the gradient is zero and the Hessian mu lam / eps P, as the
// reference regularises it.  D is evaluated as mu lam |u|^2 / (s + eps),
// the same number without the cancellation of s - eps.
// ---------------------------------------------------------------------------
struct FricLag {
    double w[4];
    V3 n;
    double lam;
};

// The frozen quantities of a classified pair at the lag state; false when
// the pair is not within dhat there.
NX_HD bool friction_lag(const DistForm& f, const V3* X, double dhat, double kappa, FricLag& L) {
    const V3 r = form_r(f, X);
    const double s = dot(r, r), sh = dhat * dhat;
    for (int k = 0; k < 4; ++k) L.w[k] = f.w[k];
    L.n = v3(0.0, 0.0, 0.0);
    L.lam = 0.0;
    if (!(s < sh) || !(s > 0.0)) return false;
    const double d = sqrt(s);
    L.n = v3(r.x / d, r.y / d, r.z / d);
    L.lam = -2.0 * d * barrier_s1(s, sh, kappa);
    return true;
}

struct FricEval {
    double e;
    V12 grad;
    double lam[2];
    V12 y[2];
};

NX_HD FricEval friction_pair(const FricLag& L, const V3* X, const V3* X0, double mu, double eps) {
    FricEval o;
    V3 dsum = v3(0.0, 0.0, 0.0);
    for (int k = 0; k < 4; ++k) dsum = dsum + L.w[k] * (X[k] - X0[k]);
    const V3 u = dsum - dot(dsum, L.n) * L.n;
    const double uu = dot(u, u), s = sqrt(uu + eps * eps), ml = mu * L.lam, un = sqrt(uu);
    o.e = ml * (uu / (s + eps));
    V3 g, t1, t2;
    if (un < 1e-12) {
        g = v3(0.0, 0.0, 0.0);
        // a tangent basis: n x (the coordinate axis least aligned with n)
        const double ax = fabs(L.n.x), ay = fabs(L.n.y), az = fabs(L.n.z);
        const V3 e = (ax <= ay && ax <= az) ? v3(1.0, 0.0, 0.0) : (ay <= az ? v3(0.0, 1.0, 0.0) : v3(0.0, 0.0, 1.0));
        const V3 c = cross(L.n, e);
        const double cn = sqrt(dot(c, c));
        t1 = v3(c.x / cn, c.y / cn, c.z / cn);
        o.lam[0] = ml / eps;
        o.lam[1] = ml / eps;
    } else {
        g = (ml / s) * u;
        t1 = v3(u.x / un, u.y / un, u.z / un);
        o.lam[0] = (ml / s) * ((eps * eps) / (s * s));
        o.lam[1] = ml / s;
    }
    t2 = cross(L.n, t1);
    for (int k = 0; k < 4; ++k) {
        o.grad.v[k] = L.w[k] * g;
        o.y[0].v[k] = L.w[k] * t1;
        o.y[1].v[k] = L.w[k] * t2;
    }
    return o;
}

// Derivatives of one frozen pair's friction point forces F_k = w_k h,
// h = mu lam u / s (friction_pair; g12 keeps its |u| < 1e-12 branch) for the
// step adjoint, lagged at the step-start points Xs (the lag state and the
// displacements' origin; fs = classify(kind, Xs)):
//   H  = dF/dX   (12 x 12, row 3k+i, column 3l+j): w_k w_l mu lam / s (P - u u^T / s^2),
//   Hs = dF/dXs  (12 x 12): through the explicit -Xs in u and through the
//        frozen weights, normal and normal force, whose derivatives follow
//        from the DistForm (du* = -g_uu^-1 g_uX dXs, dw = c du*, dr = A du* +
//        sum_k w_k dXs_k, dn = (I - n n^T) dr / d, dlam = (-2 b' - 4 d^2 b'') n.dr).
NX_HD void friction_derivs(const DistForm& fs, const V3* X, const V3* Xs, double dhat, double kappa, double mu, double eps,
                           double* g12, double* H, double* Hs) {
    const V3 r = form_r(fs, Xs);
    const double s2 = dot(r, r), sh = dhat * dhat, ds = sqrt(s2);
    const V3 n = v3(r.x / ds, r.y / ds, r.z / ds);
    const double b1 = barrier_s1(s2, sh, kappa), b2 = barrier_s2(s2, sh, kappa);
    const double lam = -2.0 * ds * b1;
    const double dlam_dd = -2.0 * b1 - 4.0 * s2 * b2;
    V3 dX[4];
    V3 dsum = v3(0.0, 0.0, 0.0);
    for (int k = 0; k < 4; ++k) {
        dX[k] = X[k] - Xs[k];
        dsum = dsum + fs.w[k] * dX[k];
    }
    const V3 u = dsum - dot(dsum, n) * n;
    const double uu = dot(u, u), s = sqrt(uu + eps * eps), ml = mu * lam;
    const V3 h = (ml / s) * u;
    const bool still = sqrt(uu) < 1e-12;
    for (int k = 0; k < 4; ++k) {
        const V3 f = still ? v3(0.0, 0.0, 0.0) : fs.w[k] * h;
        g12[3 * k] = f.x; g12[3 * k + 1] = f.y; g12[3 * k + 2] = f.z;
    }
    // M = dh/du (3 x 3) and M P
    double M[9], MP[9];
    const double cu = ml / s, cs = 1.0 / (s * s);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            const double ui = get(u, i), uj = get(u, j), ni = get(n, i), nj = get(n, j);
            M[3 * i + j] = cu * ((i == j ? 1.0 : 0.0) - ui * uj * cs);
            MP[3 * i + j] = cu * ((i == j ? 1.0 : 0.0) - ni * nj - ui * uj * cs);
        }
    for (int k = 0; k < 4; ++k)
        for (int l = 0; l < 4; ++l)
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) H[12 * (3 * k + i) + 3 * l + j] = (fs.w[k] * fs.w[l]) * MP[3 * i + j];
    // the DistForm's parameter system at Xs
    V3 a[2] = {v3(0, 0, 0), v3(0, 0, 0)};
    for (int m = 0; m < fs.nu; ++m) a[m] = fs.c[0][m] * Xs[0] + fs.c[1][m] * Xs[1] + fs.c[2][m] * Xs[2] + fs.c[3][m] * Xs[3];
    double G[2][2] = {{0, 0}, {0, 0}}, Gi[2][2] = {{0, 0}, {0, 0}};
    for (int i = 0; i < fs.nu; ++i)
        for (int j = 0; j < fs.nu; ++j) G[i][j] = 2.0 * dot(a[i], a[j]);
    if (fs.nu == 1) Gi[0][0] = 1.0 / G[0][0];
    if (fs.nu == 2) {
        const double det = G[0][0] * G[1][1] - G[0][1] * G[1][0];
        Gi[0][0] = G[1][1] / det; Gi[1][1] = G[0][0] / det; Gi[0][1] = -G[0][1] / det; Gi[1][0] = -G[1][0] / det;
    }
    for (int j = 0; j < 4; ++j)
        for (int ax = 0; ax < 3; ++ax) {
            V3 e = v3(0.0, 0.0, 0.0);
            if (ax == 0) e.x = 1.0; else if (ax == 1) e.y = 1.0; else e.z = 1.0;
            double du[2] = {0.0, 0.0};
            for (int m = 0; m < fs.nu; ++m)
                for (int q = 0; q < fs.nu; ++q)
                    du[m] -= Gi[m][q] * (2.0 * (fs.w[j] * get(a[q], ax) + fs.c[j][q] * get(r, ax)));
            double dw[4];
            for (int k = 0; k < 4; ++k) dw[k] = fs.c[k][0] * du[0] + fs.c[k][1] * du[1];
            const V3 dr = du[0] * a[0] + du[1] * a[1] + fs.w[j] * e;
            const double dd = dot(n, dr);
            const V3 dn = (1.0 / ds) * (dr - dd * n);
            const double dlam = dlam_dd * dd;
            V3 dds = (-fs.w[j]) * e;
            for (int k = 0; k < 4; ++k) dds = dds + dw[k] * dX[k];
            const V3 dU = dds - dot(dds, n) * n - dot(dsum, dn) * n - dot(dsum, n) * dn;
            V3 dh = ((mu / s) * dlam) * u;
            dh = dh + v3(M[0] * dU.x + M[1] * dU.y + M[2] * dU.z, M[3] * dU.x + M[4] * dU.y + M[5] * dU.z,
                         M[6] * dU.x + M[7] * dU.y + M[8] * dU.z);
            for (int k = 0; k < 4; ++k) {
                const V3 dF = dw[k] * h + fs.w[k] * dh;
                Hs[12 * (3 * k) + 3 * j + ax] = dF.x;
                Hs[12 * (3 * k + 1) + 3 * j + ax] = dF.y;
                Hs[12 * (3 * k + 2) + 3 * j + ax] = dF.z;
            }
        }
}

// Rigid chain: point k of the pair belongs to body side[k] (0 = body A,
// 1 = body B) at lever arm arm[k] = R r_k (world offset from the body's
// position); its DOF Jacobian is [I3, -[arm]x].  The transposed Jacobian
// maps a 12-vector of point forces to 12 body DOFs (A: 0..5, B: 6..11).
NX_HD void chain12(const V12& z, const int* side, const V3* arm, double* out12) {
    for (int i = 0; i < 12; ++i) out12[i] = 0.0;
    for (int k = 0; k < 4; ++k) {
        double* o = out12 + 6 * side[k];
        const V3 t = cross(arm[k], z.v[k]);
        o[0] += z.v[k].x; o[1] += z.v[k].y; o[2] += z.v[k].z;
        o[3] += t.x; o[4] += t.y; o[5] += t.z;
    }
}

// Rotations of the iterate are R = Exp(theta) R0 (rot_gt).  A point's world
// offset a = Exp(theta) R0 r moves by da = -[a]x J_l(theta) dtheta, so the
// exact gradient of an energy of world points with respect to theta is
// J_l(theta)^T sum_k a_k x g_k = J_r(theta) (torque): the lever-arm torque
// (chain12) times the right Jacobian of SO(3),
//   J_r(theta) = I - c1 [theta]x + c2 [theta]x^2,
//   c1 = (1 - cos phi) / phi^2,  c2 = (phi - sin phi) / phi^3,  phi = |theta|,
// with the series below phi = 1e-2 (truncation far below rounding).
NX_HD void jr_coeffs(double phi, double& c1, double& c2) {
    const double p2 = phi * phi;
    if (phi < 1e-2) {
        c1 = 0.5 - p2 * (1.0 / 24.0) + (p2 * p2) * (1.0 / 720.0);
        c2 = 1.0 / 6.0 - p2 * (1.0 / 120.0) + (p2 * p2) * (1.0 / 5040.0);
        return;
    }
    double sn, cs;
    nxm::sincos(phi, &sn, &cs);
    c1 = (1.0 - cs) / p2;
    c2 = (phi - sn) / (p2 * phi);
}
// J_r(theta) v
NX_HD V3 jr_apply(V3 th, V3 v) {
    double c1, c2;
    jr_coeffs(sqrt(dot(th, th)), c1, c2);
    const V3 tv = cross(th, v);
    return v - c1 * tv + c2 * cross(th, tv);
}
// chain12 with the exact rotation derivative: the rotational parts of body
// A (out12[3..5]) and B (out12[9..11]) multiplied by J_r(theta_A), J_r(theta_B)
NX_HD void chain12_exact(const V12& z, const int* side, const V3* arm, V3 thA, V3 thB, double* out12) {
    chain12(z, side, arm, out12);
    const V3 ta = jr_apply(thA, v3(out12[3], out12[4], out12[5]));
    const V3 tb = jr_apply(thB, v3(out12[9], out12[10], out12[11]));
    out12[3] = ta.x; out12[4] = ta.y; out12[5] = ta.z;
    out12[9] = tb.x; out12[10] = tb.y; out12[11] = tb.z;
}

// ---- step adjoint helpers -------------------------------------------------
// c1, c2 of J_r and their derivatives over phi: d1 = c1'(phi) / phi,
// d2 = c2'(phi) / phi (series below phi = 1e-2).
NX_HD void jr_coeffs_d(double phi, double& c1, double& c2, double& d1, double& d2) {
    const double p2 = phi * phi;
    if (phi < 1e-2) {
        const double p4 = p2 * p2;
        c1 = 0.5 - p2 * (1.0 / 24.0) + p4 * (1.0 / 720.0);
        c2 = 1.0 / 6.0 - p2 * (1.0 / 120.0) + p4 * (1.0 / 5040.0);
        d1 = -2.0 / 24.0 + p2 * (4.0 / 720.0) - p4 * (6.0 / 40320.0);
        d2 = -2.0 / 120.0 + p2 * (4.0 / 5040.0) - p4 * (6.0 / 362880.0);
        return;
    }
    double sn, cs;
    nxm::sincos(phi, &sn, &cs);
    const double p3 = p2 * phi, p4 = p2 * p2;
    c1 = (1.0 - cs) / p2;
    c2 = (phi - sn) / p3;
    d1 = sn / p3 - 2.0 * (1.0 - cs) / p4;
    d2 = (1.0 - cs) / p4 - 3.0 * (phi - sn) / (p4 * phi);
}
// 3 x 3 row-major helpers
NX_HD void m3_skew(V3 v, double* S) {
    S[0] = 0.0; S[1] = -v.z; S[2] = v.y;
    S[3] = v.z; S[4] = 0.0; S[5] = -v.x;
    S[6] = -v.y; S[7] = v.x; S[8] = 0.0;
}
NX_HD void m3_mul(const double* A, const double* B, double* C) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) C[3 * i + j] = A[3 * i] * B[j] + A[3 * i + 1] * B[3 + j] + A[3 * i + 2] * B[6 + j];
}
// Exp(theta) as a matrix: I + sinc [t]x + c1 [t]x^2, and J_l(theta) =
// I + c1 [t]x + c2 [t]x^2 (J_r = J_l^T).
NX_HD void rot_exp_mats(V3 th, double* R, double* Jl) {
    const double phi = sqrt(dot(th, th));
    double c1, c2, d1, d2;
    jr_coeffs_d(phi, c1, c2, d1, d2);
    double sinc;
    if (phi < 1e-2) { const double p2 = phi * phi; sinc = 1.0 - p2 * (1.0 / 6.0) + (p2 * p2) * (1.0 / 120.0); }
    else { double sn, cs; nxm::sincos(phi, &sn, &cs); sinc = sn / phi; }
    double S[9], S2[9];
    m3_skew(th, S);
    m3_mul(S, S, S2);
    for (int e = 0; e < 9; ++e) {
        const double id = (e % 4 == 0) ? 1.0 : 0.0;
        R[e] = id + sinc * S[e] + c1 * S2[e];
        Jl[e] = id + c1 * S[e] + c2 * S2[e];
    }
}
// M = d(J_r(theta) tau)/dtheta at fixed tau, row-major:
//   -(t x tau) (d1 t)^T + c1 [tau]x + (t x (t x tau)) (d2 t)^T
//   + c2 ((t . tau) I + t tau^T - 2 tau t^T)
NX_HD void jr_torque_derivative(V3 th, V3 tau, double* M) {
    double c1, c2, d1, d2;
    jr_coeffs_d(sqrt(dot(th, th)), c1, c2, d1, d2);
    const V3 tt = cross(th, tau), ttt = cross(th, tt);
    const double td = dot(th, tau);
    const double t[3] = {th.x, th.y, th.z}, u[3] = {tau.x, tau.y, tau.z};
    const double a[3] = {tt.x, tt.y, tt.z}, b[3] = {ttt.x, ttt.y, ttt.z};
    double S[9];
    m3_skew(tau, S);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            M[3 * i + j] = -(a[i] * (d1 * t[j])) + c1 * S[3 * i + j] + b[i] * (d2 * t[j]) +
                           c2 * ((i == j ? td : 0.0) + t[i] * u[j] - 2.0 * (u[i] * t[j]));
}

// Additive CCD along linear point trajectories X + t P, t in [0, t_max]:
// the relative motion of the pair (common translation removed) changes the
// distance by at most lp per unit t, so from distance d at t every point of
// [t, t + dl], dl = 0.9 (d - g) / lp, keeps the distance above g = eta d(0).
// One round evaluates the distance d_j at the samples t_j = t + j dl,
// j = 1..kAccdLookahead, and advances to the first sample with
// d_j < g + 0.9 (d - g) (from a sample at or above that bound the next dl
// keeps the distance above g), or to the last sample; a sample reached that
// way at or past t_max returns t_max.  A contact that slides without
// closing in advances kAccdLookahead steps per round instead of one.  At
// most max_iter rounds; every returned t keeps the distance >= g on [0, t].
// The sample loop below is sequential; the device evaluates a round's
// samples in the lanes of one warp (accd_round_warp) with the same
// arithmetic and the same choice.
constexpr int kAccdLookahead = 32;

NX_HD double accd_lipschitz(int kind, const V3* P0) {
    V3 P[4];
    const V3 mean = 0.25 * ((P0[0] + P0[1]) + (P0[2] + P0[3]));
    for (int k = 0; k < 4; ++k) P[k] = P0[k] - mean;
    if (kind == kPairPT) return norm(P[0]) + dmax(norm(P[1]), dmax(norm(P[2]), norm(P[3])));
    return dmax(norm(P[0]), norm(P[1])) + dmax(norm(P[2]), norm(P[3]));
}
NX_HD double accd_distance(int kind, const V3* X0, const V3* P0, double t) {
    V3 X[4];
    for (int k = 0; k < 4; ++k) X[k] = X0[k] + t * P0[k];
    return sqrt(dist2(kind, X));
}

// The points moving on their chords: X_k(t) = X0_k + t P0_k.
struct ChordMotion {
    V3 X0[4], P0[4];
    int kind;
    NX_HD double lipschitz() const { return accd_lipschitz(kind, P0); }
    NX_HD double distance(double t) const { return accd_distance(kind, X0, P0, t); }
};

// The points moving rigidly with their bodies along the iterates x + t dx:
// point k (body-local v_k, body side[k]) at t is
//   p + t dp + rot(Exp(theta + t dtheta) q0, v_k),
// the world-vertex formula at the pose x + t dx, so the pose of a line-search
// trial at alpha is this motion at t = alpha bit for bit.  Its speed is at
// most |dp| + |dtheta| |v_k| (|J_l(theta)| <= 1); with the common velocity
// dp_A removed, the distance changes at most at
//   max_{k on A} |dtheta_A| |v_k| + max_{k on B} (|dp_B - dp_A| + |dtheta_B| |v_k|).
struct ArcBody {
    V3 p, dp, th, dth;
    Q q0;
};
struct ArcMotion {
    ArcBody b[2];
    V3 v[4];
    int side[4];
    int kind;
    NX_HD void points(double t, V3* X) const {
        V3 pp[2];
        Q q[2];
        for (int s = 0; s < 2; ++s) {
            pp[s] = b[s].p + t * b[s].dp;
            q[s] = rot_gt(b[s].q0, b[s].th + t * b[s].dth);
        }
        for (int k = 0; k < 4; ++k) X[k] = pp[side[k]] + qrot(q[side[k]], v[k]);
    }
    NX_HD double lipschitz() const {
        const double wa = norm(b[0].dth), wb = norm(b[1].dth), tb = norm(b[1].dp - b[0].dp);
        double la = 0.0, lb = 0.0;
        for (int k = 0; k < 4; ++k) {
            if (side[k] == 0) la = dmax(la, wa * norm(v[k]));
            else lb = dmax(lb, tb + wb * norm(v[k]));
        }
        return la + lb;
    }
    NX_HD double distance(double t) const {
        V3 X[4];
        points(t, X);
        return sqrt(dist2(kind, X));
    }
};

// Additive CCD along a motion M (ChordMotion or ArcMotion).
template <typename M>
NX_HD double accd_toi_motion(int kind, const M& m, double t_max, double eta, int max_iter, int* iters) {
    const double lp = m.lipschitz();
    if (iters) *iters = 0;
    const double d0 = m.distance(0.0);
    if (!(lp > 0.0)) return t_max;
    if (!(d0 > 0.0)) return 0.0;
    const double g = eta * d0;
    double t = 0.0, d = d0;
    for (int it = 0; it < max_iter; ++it) {
        if (iters) *iters = it + 1;
        const double dl = 0.9 * (d - g) / lp;
        if (t + dl >= t_max) return t_max;
        if (!(dl > 1e-12 * t_max)) return t;
        const double thr = g + 0.9 * (d - g);
        double tn = t, dn = d;
        for (int j = 1; j <= kAccdLookahead; ++j) {
            const double tj = t + (double)j * dl;
            if (tj >= t_max) return t_max;
            const double dj = m.distance(tj);
            tn = tj;
            dn = dj;
            if (!(dj >= thr)) break;
        }
        t = tn;
        d = dn;
    }
    return t;
}

NX_HD double accd_toi(int kind, const V3* X0, const V3* P0, double t_max, double eta, int max_iter, int* iters) {
    ChordMotion m;
    for (int k = 0; k < 4; ++k) { m.X0[k] = X0[k]; m.P0[k] = P0[k]; }
    m.kind = kind;
    return accd_toi_motion(kind, m, t_max, eta, max_iter, iters);
}

// Swept boxes for the arc motion: a point's rotation part moves at most
// |dtheta| |v| per unit t, so it stays within |dtheta| |v| / 2 of one of its
// ends (the translation part is linear, exact on the chord); the box of a
// body's endpoints padded by |dtheta_b| r_b / 2 (r_b its largest |v|)
// contains its points' arcs.
NX_HD double arc_box_pad(V3 dth, double r_body) { return 0.5 * (norm(dth) * r_body); }

}  // namespace ipc
}  // namespace nx
