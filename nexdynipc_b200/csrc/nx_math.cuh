// nx_math.cuh — FP64 vector / quaternion algebra for the contact step.
//
// Operation order follows the Eigen 3 expressions the reference evaluates
// (nexdynipc uses Eigen::Quaterniond / Vector3d throughout):
//   q * v        = v + w*t + vec x t,  t = 2 (vec x v)          (Quaternion::_transformVector)
//   a * b        = Hamilton product, terms left to right
//   normalized() = coeffs / sqrt(squaredNorm), coeffs stored (x,y,z,w)
//   AngleAxis(angle, axis) -> (cos(angle/2), sin(angle/2) axis)
//   Quaternion -> AngleAxis: angle = 2 atan2(|vec|, |w|), axis = vec / (+-|vec|)
// Every kernel is compiled with --fmad=false, so each product and sum is
// separately rounded, as on the host side; sin, cos, atan2 and log come from
// nx_libm.h, the same code the CPU oracle uses.
#pragma once

#include <cmath>
#include <cstdint>

#include "nx_libm.h"

#ifdef __CUDACC__
#define NX_HD __host__ __device__ __forceinline__
#define NX_UNROLL _Pragma("unroll")
#else
#define NX_HD inline
#define NX_UNROLL
#endif

namespace nx {

struct V3 { double x, y, z; };
struct Q { double w, x, y, z; };

NX_HD V3 v3(double x, double y, double z) { V3 r; r.x = x; r.y = y; r.z = z; return r; }
NX_HD V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
NX_HD V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
NX_HD V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
NX_HD V3 operator*(double s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
NX_HD V3 operator*(V3 a, double s) { return v3(a.x * s, a.y * s, a.z * s); }
NX_HD V3 operator/(V3 a, double s) { return v3(a.x / s, a.y / s, a.z / s); }
NX_HD double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
NX_HD V3 cross(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
NX_HD double sqnorm(V3 a) { return dot(a, a); }
NX_HD double norm(V3 a) { return sqrt(sqnorm(a)); }
NX_HD V3 normalized(V3 a) {
    const double z = sqnorm(a);
    return z > 0.0 ? a / sqrt(z) : a;
}
NX_HD double get(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
NX_HD double dmin(double a, double b) { return (b < a) ? b : a; }   // std::min
NX_HD double dmax(double a, double b) { return (a < b) ? b : a; }   // std::max
NX_HD V3 cwmin(V3 a, V3 b) { return v3(dmin(a.x, b.x), dmin(a.y, b.y), dmin(a.z, b.z)); }
NX_HD V3 cwmax(V3 a, V3 b) { return v3(dmax(a.x, b.x), dmax(a.y, b.y), dmax(a.z, b.z)); }
NX_HD V3 ld3(const double* p) { return v3(p[0], p[1], p[2]); }
NX_HD void st3(double* p, V3 v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }

NX_HD Q q4(double w, double x, double y, double z) { Q q; q.w = w; q.x = x; q.y = y; q.z = z; return q; }
NX_HD Q ldq(const double* p) { return q4(p[0], p[1], p[2], p[3]); }
NX_HD void stq(double* p, Q q) { p[0] = q.w; p[1] = q.x; p[2] = q.y; p[3] = q.z; }
NX_HD V3 qvec(Q q) { return v3(q.x, q.y, q.z); }
NX_HD Q qmul(Q a, Q b) {
    return q4(a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z,
              a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
              a.w * b.y + a.y * b.w + a.z * b.x - a.x * b.z,
              a.w * b.z + a.z * b.w + a.x * b.y - a.y * b.x);
}
NX_HD V3 qrot(Q q, V3 v) {
    V3 uv = cross(qvec(q), v);
    uv = uv + uv;
    return v + q.w * uv + cross(qvec(q), uv);
}
NX_HD Q qconj(Q q) { return q4(q.w, -q.x, -q.y, -q.z); }
NX_HD Q qnormalized(Q q) {
    const double n2 = (q.x * q.x + q.z * q.z) + (q.y * q.y + q.w * q.w);
    if (!(n2 > 0.0)) return q;
    const double n = sqrt(n2);
    return q4(q.w / n, q.x / n, q.y / n, q.z / n);
}
NX_HD Q q_from_angle_axis(double angle, V3 axis) {
    const double ha = 0.5 * angle;
    double s, c;
    nxm::sincos(ha, &s, &c);
    return q4(c, s * axis.x, s * axis.y, s * axis.z);
}
NX_HD void q_to_angle_axis(Q q, double& angle, V3& axis) {
    double n = norm(qvec(q));
    if (n != 0.0) {
        angle = 2.0 * nxm::atan2(n, fabs(q.w));
        if (q.w < 0.0) n = -n;
        axis = qvec(q) / n;
    } else {
        angle = 0.0;
        axis = v3(1, 0, 0);
    }
}
// JointPrimitives::updateRotation (NexDynIPC/Dynamics/Joints/JointPrimitives.h:11-19): '<' threshold
NX_HD Q rot_joint(Q q_ref, V3 th) {
    const double a = norm(th);
    if (a < 1e-10) return q_ref;
    return qnormalized(qmul(q_from_angle_axis(a, th / a), q_ref));
}
// FrictionForm::getBodyState / detectContactsAtState / step write-back: '>' threshold
// (src/Dynamics/Forms/FrictionForm.cpp:206-224, src/Dynamics/IPCSolver.cpp:618-626)
NX_HD Q rot_gt(Q q_ref, V3 th) {
    const double a = norm(th);
    if (a > 1e-10) return qnormalized(qmul(q_from_angle_axis(a, th / a), q_ref));
    return q_ref;
}

struct M3 { double m[9]; };
NX_HD double& at(M3& A, int r, int c) { return A.m[3 * r + c]; }
NX_HD double at(const M3& A, int r, int c) { return A.m[3 * r + c]; }
NX_HD M3 cross_mat(V3 v) {
    M3 M;
    M.m[0] = 0.0; M.m[1] = -v.z; M.m[2] = v.y;
    M.m[3] = v.z; M.m[4] = 0.0; M.m[5] = -v.x;
    M.m[6] = -v.y; M.m[7] = v.x; M.m[8] = 0.0;
    return M;
}
NX_HD M3 mat_mul(const M3& A, const M3& B) {
    M3 C;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            C.m[3 * i + j] = A.m[3 * i] * B.m[j] + A.m[3 * i + 1] * B.m[3 + j] + A.m[3 * i + 2] * B.m[6 + j];
    return C;
}
NX_HD V3 mat_vec(const double* A, V3 v) {
    return v3(A[0] * v.x + A[1] * v.y + A[2] * v.z, A[3] * v.x + A[4] * v.y + A[5] * v.z,
              A[6] * v.x + A[7] * v.y + A[8] * v.z);
}

// AABB helpers (NexDynIPC/Physics/Geometry/AABB.h), boxes as mn[3], mx[3].
struct Box { V3 mn, mx; };
NX_HD Box box_empty() {
    Box b;
    b.mn = v3(1.7976931348623157e308, 1.7976931348623157e308, 1.7976931348623157e308);
    b.mx = v3(-1.7976931348623157e308, -1.7976931348623157e308, -1.7976931348623157e308);
    return b;
}
NX_HD void box_expand(Box& b, V3 p) { b.mn = cwmin(b.mn, p); b.mx = cwmax(b.mx, p); }
NX_HD Box box_inflated(Box b, double m) {
    Box r;
    r.mn = v3(b.mn.x - m, b.mn.y - m, b.mn.z - m);
    r.mx = v3(b.mx.x + m, b.mx.y + m, b.mx.z + m);
    return r;
}
NX_HD bool box_intersects(const Box& a, const Box& o) {
    return a.mn.x <= o.mx.x && a.mn.y <= o.mx.y && a.mn.z <= o.mx.z && a.mx.x >= o.mn.x && a.mx.y >= o.mn.y &&
           a.mx.z >= o.mn.z;
}
NX_HD double max3(double a, double b, double c) { return dmax(dmax(a, b), c); }
// aabb_distance (src/Physics/Contact/ContactAssembler.cpp:45-55)
NX_HD double box_distance(const Box& a, const Box& b) {
    const double dx = max3(0.0, a.mn.x - b.mx.x, b.mn.x - a.mx.x);
    const double dy = max3(0.0, a.mn.y - b.mx.y, b.mn.y - a.mx.y);
    const double dz = max3(0.0, a.mn.z - b.mx.z, b.mn.z - a.mx.z);
    return sqrt(dx * dx + dy * dy + dz * dz);
}
// point_aabb_distance (ContactAssembler.cpp:57-65)
NX_HD double point_box_distance(V3 p, const Box& b) {
    const double dx = max3(b.mn.x - p.x, 0.0, p.x - b.mx.x);
    const double dy = max3(b.mn.y - p.y, 0.0, p.y - b.mx.y);
    const double dz = max3(b.mn.z - p.z, 0.0, p.z - b.mx.z);
    return sqrt(dx * dx + dy * dy + dz * dz);
}
// transform_local_aabb (ContactAssembler.cpp:22-43)
NX_HD Box transform_local_box(V3 mn, V3 mx, V3 pos, Q q) {
    Box b = box_empty();
    for (int ix = 0; ix < 2; ++ix)
        for (int iy = 0; iy < 2; ++iy)
            for (int iz = 0; iz < 2; ++iz) {
                const V3 c = v3(ix ? mx.x : mn.x, iy ? mx.y : mn.y, iz ? mx.z : mn.z);
                box_expand(b, pos + qrot(q, c));
            }
    return b;
}

// BarrierPotential (src/Physics/Contact/Barrier.cpp:11-46)
NX_HD double barrier_value(double d, double dh, double k) {
    if (d >= dh) return 0.0;
    if (d <= 0.0) return INFINITY;
    const double r = d / dh;
    return -k * (d - dh) * (d - dh) * nxm::log(r);
}
NX_HD double barrier_gradient(double d, double dh, double k) {
    if (d >= dh) return 0.0;
    if (d <= 0.0) return -INFINITY;
    const double diff = d - dh;
    const double lr = nxm::log(d / dh);
    return -k * (2 * diff * lr + diff * diff / d);
}
NX_HD double barrier_hessian(double d, double dh, double k) {
    if (d >= dh) return 0.0;
    if (d <= 0.0) return INFINITY;
    const double diff = d - dh;
    const double lr = nxm::log(d / dh);
    return -k * (2 * lr + 4 * diff / d - (diff * diff) / (d * d));
}

}  // namespace nx
