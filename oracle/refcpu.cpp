// refcpu.cpp — CPU oracle (test infrastructure, never shipped as the product).
//
// A plain C++17 restatement of NexDynIPC's IPCSolver::step and everything it
// calls (paths below are relative to the NexDynIPC project root).  Eigen and
// Boost are absent on this machine, so the small linear algebra the reference
// takes from them is restated here from the published methods:
//   * Eigen 3 Quaternion: Hamilton product, q*v as v + w*t + vec x t with
//     t = 2 vec x v, normalized() as coeffs / sqrt(squaredNorm),
//     AngleAxis <-> Quaternion conversions (half-angle sin/cos; 2*atan2(|v|,|w|)).
//   * Eigen SimplicialLDLT: any exact LDL^T of the assembled sparse Hessian;
//     here a dense LDL^T per connected block component in ascending DOF order
//     (the reference uses an AMD ordering; its rounding is not pinned by any
//     reference test).  It fails, like Eigen, only on an exactly zero pivot.
//   * Boost.Interval: outward-rounded intervals (nextafter based).
// libstdc++ (GCC 13, on this machine) supplies std::nth_element and std::sort
// exactly as the reference calls them.
//
// Build: oracle/build.sh (g++ -O3 -ffp-contract=off -fopenmp -shared).

#include "refcpu.h"

// Elementary functions: the same portable implementations the device code
// uses (Cody-Waite reduction + Taylor series), so the two sides round alike.
#include "../nexdynipc_b200/csrc/nx_libm.h"

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <memory>
#include <numeric>
#include <stack>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif


// primitive-pair barrier of ipc_cpu.cpp with its block structure, and its
// lagged friction (IpcFricCtx: the frozen pairs, built at the evaluation
// after ipc_fric_rebuild)
struct IpcFricCtx;
IpcFricCtx* ipc_fric_new(double mu, double eps);
void ipc_fric_free(IpcFricCtx* f);
void ipc_fric_rebuild(IpcFricCtx* f);
int64_t ipc_fric_count(const IpcFricCtx* f);
double ipc_fric_energy(const IpcFricCtx* f);
int ipc_barrier_cpu(nxo_world* w, const double* x, double dhat, double kappa, double* energy, double* grad, double* H,
                    std::vector<std::pair<int, int>>* blocks, int64_t* n_pairs, int64_t* n_active, IpcFricCtx* fr);

namespace {

constexpr double kInf = std::numeric_limits<double>::infinity();

// ---------------------------------------------------------------------------
// Small vector / quaternion algebra (Eigen semantics, see file header).
// ---------------------------------------------------------------------------
struct V3 {
    double x = 0, y = 0, z = 0;
    double operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    double& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
};
inline V3 mk(double x, double y, double z) { V3 v; v.x = x; v.y = y; v.z = z; return v; }
inline V3 operator+(V3 a, V3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 operator-(V3 a, V3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 operator-(V3 a) { return mk(-a.x, -a.y, -a.z); }
inline V3 operator*(double s, V3 a) { return mk(s * a.x, s * a.y, s * a.z); }
inline V3 operator*(V3 a, double s) { return mk(a.x * s, a.y * s, a.z * s); }
inline V3 operator/(V3 a, double s) { return mk(a.x / s, a.y / s, a.z / s); }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline double sqnorm(V3 a) { return dot(a, a); }
inline double norm(V3 a) { return std::sqrt(sqnorm(a)); }
inline V3 normalized(V3 a) {
    const double z = sqnorm(a);
    return z > 0.0 ? a / std::sqrt(z) : a;
}
inline V3 cwmin(V3 a, V3 b) { return mk(std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z)); }
inline V3 cwmax(V3 a, V3 b) { return mk(std::max(a.x, b.x), std::max(a.y, b.y), std::max(a.z, b.z)); }

struct Q {
    double w = 1, x = 0, y = 0, z = 0;
};
inline Q mkq(double w, double x, double y, double z) { Q q; q.w = w; q.x = x; q.y = y; q.z = z; return q; }
inline V3 qvec(Q q) { return mk(q.x, q.y, q.z); }
inline Q qmul(Q a, Q b) {
    return mkq(a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z,
               a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
               a.w * b.y + a.y * b.w + a.z * b.x - a.x * b.z,
               a.w * b.z + a.z * b.w + a.x * b.y - a.y * b.x);
}
inline V3 qrot(Q q, V3 v) {
    V3 uv = cross(qvec(q), v);
    uv = uv + uv;
    return v + q.w * uv + cross(qvec(q), uv);
}
inline Q qconj(Q q) { return mkq(q.w, -q.x, -q.y, -q.z); }
inline Q qnormalized(Q q) {
    // coeffs() are stored (x, y, z, w); the 4-term sum pairs (x,z) and (y,w)
    // the way a 2-wide packet reduction of that storage does.
    const double n2 = (q.x * q.x + q.z * q.z) + (q.y * q.y + q.w * q.w);
    if (!(n2 > 0.0)) return q;
    const double n = std::sqrt(n2);
    return mkq(q.w / n, q.x / n, q.y / n, q.z / n);
}
inline Q q_from_angle_axis(double angle, V3 axis) {
    const double ha = 0.5 * angle;
    double s, c;
    nxm::sincos(ha, &s, &c);
    return mkq(c, s * axis.x, s * axis.y, s * axis.z);
}
inline void q_to_angle_axis(Q q, double& angle, V3& axis) {
    double n = norm(qvec(q));
    if (n != 0.0) {
        angle = 2.0 * nxm::atan2(n, std::fabs(q.w));
        if (q.w < 0.0) n = -n;
        axis = qvec(q) / n;
    } else {
        angle = 0.0;
        axis = mk(1, 0, 0);
    }
}
// JointPrimitives::updateRotation (NexDynIPC/Dynamics/Joints/JointPrimitives.h:11-19)
inline Q update_rotation_joint(Q q_ref, V3 theta) {
    const double angle = norm(theta);
    if (angle < 1e-10) return q_ref;
    const V3 axis = theta / angle;
    return qnormalized(qmul(q_from_angle_axis(angle, axis), q_ref));
}
// FrictionForm::getBodyState / detectContactsAtState / step write-back use '>'
// (FrictionForm.cpp:206-224, IPCSolver.cpp:618-626, IPCSolver.cpp:1187-1192).
inline Q update_rotation_gt(Q q_ref, V3 theta) {
    const double angle = norm(theta);
    if (angle > 1e-10) {
        const V3 axis = theta / angle;
        return qnormalized(qmul(q_from_angle_axis(angle, axis), q_ref));
    }
    return q_ref;
}

struct M3 {
    double m[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    double operator()(int r, int c) const { return m[3 * r + c]; }
    double& operator()(int r, int c) { return m[3 * r + c]; }
};
inline V3 mul(const M3& A, V3 v) {
    return mk(A(0, 0) * v.x + A(0, 1) * v.y + A(0, 2) * v.z,
              A(1, 0) * v.x + A(1, 1) * v.y + A(1, 2) * v.z,
              A(2, 0) * v.x + A(2, 1) * v.y + A(2, 2) * v.z);
}

// ---------------------------------------------------------------------------
// AABB (NexDynIPC/Physics/Geometry/AABB.h:15-259)
// ---------------------------------------------------------------------------
struct AABB {
    V3 mn = mk(std::numeric_limits<double>::max(), std::numeric_limits<double>::max(),
               std::numeric_limits<double>::max());
    V3 mx = mk(std::numeric_limits<double>::lowest(), std::numeric_limits<double>::lowest(),
               std::numeric_limits<double>::lowest());
    AABB() = default;
    AABB(V3 a, V3 b) : mn(a), mx(b) {}
    V3 center() const { return (mn + mx) * 0.5; }
    V3 extent() const { return mx - mn; }
    double surfaceArea() const {
        V3 e = extent();
        return 2.0 * (e.x * e.y + e.y * e.z + e.z * e.x);
    }
    void expand(V3 p) { mn = cwmin(mn, p); mx = cwmax(mx, p); }
    void expand(const AABB& o) { mn = cwmin(mn, o.mn); mx = cwmax(mx, o.mx); }
    AABB merged(const AABB& o) const { return AABB(cwmin(mn, o.mn), cwmax(mx, o.mx)); }
    bool intersects(const AABB& o) const {
        return mn.x <= o.mx.x && mn.y <= o.mx.y && mn.z <= o.mx.z && mx.x >= o.mn.x &&
               mx.y >= o.mn.y && mx.z >= o.mn.z;
    }
    AABB inflated(double m) const {
        return AABB(mk(mn.x - m, mn.y - m, mn.z - m), mk(mx.x + m, mx.y + m, mx.z + m));
    }
    int maxExtentAxis() const {
        V3 e = extent();
        if (e.x >= e.y && e.x >= e.z) return 0;
        if (e.y >= e.z) return 1;
        return 2;
    }
};

// ---------------------------------------------------------------------------
// BVH (src/Physics/Geometry/BVH.cpp:19-362), built and queried as written.
// ---------------------------------------------------------------------------
struct BVH {
    struct Node { AABB bbox; int left = -1, right = -1, parent = -1, primitive = -1;
                   bool isLeaf() const { return left < 0 && right < 0; } };
    std::vector<Node> nodes;
    int root = -1;

    void init(const std::vector<AABB>& aabbs) {
        nodes.clear(); root = -1;
        if (aabbs.empty()) return;
        std::vector<int> prims(aabbs.size());
        for (size_t i = 0; i < aabbs.size(); ++i) prims[i] = (int)i;
        nodes.reserve(2 * aabbs.size() - 1);
        root = build(prims, aabbs);
    }
    int findSAHSplit(const std::vector<int>& prims, const std::vector<AABB>& aabbs, int axis) {
        const int numBins = 16;
        const int n = (int)prims.size();
        double minC = std::numeric_limits<double>::max(), maxC = std::numeric_limits<double>::lowest();
        for (int p : prims) { double c = aabbs[p].center()[axis]; minC = std::min(minC, c); maxC = std::max(maxC, c); }
        if (maxC - minC < 1e-10) return n / 2;
        std::vector<AABB> binA(numBins);
        std::vector<int> binC(numBins, 0);
        const double bw = (maxC - minC) / numBins;
        for (int p : prims) {
            double c = aabbs[p].center()[axis];
            int b = std::min(numBins - 1, (int)((c - minC) / bw));
            binA[b].expand(aabbs[p]); binC[b]++;
        }
        std::vector<double> la(numBins, 0), ra(numBins, 0);
        std::vector<int> lc(numBins, 0), rc(numBins, 0);
        AABB lb; int lt = 0;
        for (int i = 0; i < numBins; ++i) { lb.expand(binA[i]); lt += binC[i]; la[i] = lb.surfaceArea(); lc[i] = lt; }
        AABB rb; int rt = 0;
        for (int i = numBins - 1; i >= 0; --i) { rb.expand(binA[i]); rt += binC[i]; ra[i] = rb.surfaceArea(); rc[i] = rt; }
        double best = std::numeric_limits<double>::max(); int split = n / 2;
        for (int i = 0; i < numBins - 1; ++i) {
            if (lc[i] == 0 || rc[i + 1] == 0) continue;
            double cost = la[i] * lc[i] + ra[i + 1] * rc[i + 1];
            if (cost < best) { best = cost; split = lc[i]; }
        }
        return split;
    }
    int build(std::vector<int>& prims, const std::vector<AABB>& aabbs) {
        if (prims.empty()) return -1;
        int id = (int)nodes.size();
        nodes.push_back(Node());
        if (prims.size() == 1) { nodes[id].bbox = aabbs[prims[0]]; nodes[id].primitive = prims[0]; return id; }
        AABB cb;
        for (int p : prims) cb.expand(aabbs[p].center());
        int axis = cb.maxExtentAxis();
        int mid;
        if (cb.extent()[axis] < 1e-10) {
            mid = (int)prims.size() / 2;
        } else {
            mid = findSAHSplit(prims, aabbs, axis);
            if (mid <= 0 || mid >= (int)prims.size()) {
                mid = (int)prims.size() / 2;
                std::nth_element(prims.begin(), prims.begin() + mid, prims.end(),
                                 [&](int a, int b) { return aabbs[a].center()[axis] < aabbs[b].center()[axis]; });
            }
        }
        std::vector<int> lp(prims.begin(), prims.begin() + mid), rp(prims.begin() + mid, prims.end());
        int l = build(lp, aabbs), r = build(rp, aabbs);
        nodes[id].left = l; nodes[id].right = r;
        nodes[id].bbox = nodes[l].bbox.merged(nodes[r].bbox);
        nodes[l].parent = id; nodes[r].parent = id;
        return id;
    }
    void intersectBox(const AABB& q, std::vector<unsigned>& out) const {
        out.clear();
        if (root < 0) return;
        std::stack<int> st; st.push(root);
        while (!st.empty()) {
            int id = st.top(); st.pop();
            const Node& nd = nodes[id];
            if (!nd.bbox.intersects(q)) continue;
            if (nd.isLeaf()) out.push_back((unsigned)nd.primitive);
            else { if (nd.left >= 0) st.push(nd.left); if (nd.right >= 0) st.push(nd.right); }
        }
    }
};

// ---------------------------------------------------------------------------
// World data
// ---------------------------------------------------------------------------
struct Mesh {
    std::vector<V3> V;
    std::vector<std::array<int, 3>> F;
    std::vector<std::array<int, 2>> E;   // unique edges, built once (see build_unique_edges)
    V3 aabb_min, aabb_max;               // MeshShape ctor (src/Physics/Geometry/MeshShape.cpp:6-11)
};

struct Body {
    int id = -1;
    V3 position, velocity, angular_velocity, linear_acceleration, angular_acceleration;
    Q orientation;
    double mass = 1.0;
    M3 inertia;
    int mesh = -1;
};

struct Joint {
    int type = 0;
    int bodyA_id = -1, bodyB_id = -1;
    V3 anchorA, anchorB, axisA, axisB;   // hinge / spherical
    V3 target_pos; Q target_ori;         // fixed
    V3 axis; double min_angle = 0, max_angle = 0;  // angle limit (axis normalised)
    double mu = 1e8;
    std::vector<double> lambda;
    // updateState
    int gA = -1, gB = -1;
    V3 pA_ref, pB_ref; Q qA_ref, qB_ref;
    V3 uA, vA, uB, vB;                   // prismatic / cylindrical bases (computeBasis)
    double min_dist = 0, max_dist = 0;   // distance limit
    int dim() const {
        if (type == NXD_JOINT_HINGE || type == NXD_JOINT_FIXED) return 6;
        if (type == NXD_JOINT_PRISMATIC) return 5;
        if (type == NXD_JOINT_CYLINDRICAL) return 4;
        return type == NXD_JOINT_SPHERICAL ? 3 : 2;
    }
    bool is_limit() const { return type == NXD_JOINT_ANGLE_LIMIT || type == NXD_JOINT_DISTANCE_LIMIT; }
};

// Control form of World::forms.  The velocity and position drives use axis,
// kv (kp), v_target (target position), max_torque (max force), delay
// (deadzone) and delay_tau; the force drive force / torque; the spring
// rest / k / c.
struct Drive {
    int kind = NXD_DRIVE_ANGULAR_VELOCITY;
    int bodyA = -1, bodyB = -1;    // world indices (-1: none)
    V3 axis; double kv = 0, v_target = 0, max_torque = kInf, delay = 0, delay_tau = 0;
    V3 force, torque;
    double rest = 0, k = 0, c = 0;
    double dt = 0.01;
    int gA = -1, gB = -1;
    V3 prevA, prevB; bool has_prev = false;
    bool filter_init = false; double filtered = 0;
};

struct Contact {
    int bodyA = 0, bodyB = 0, type = 0, primA = 0, primB = 0;
    V3 point, normal;
    double distance = 0;
};

struct Trip { int r, c; double v; };

struct BodyContactMesh {
    int body_id = -1, world_index = -1;
    const Mesh* mesh = nullptr;
    V3 world_position; Q world_orientation;
    AABB world_aabb;
};

struct CandVV { int b0, b1, v0, v1; };
struct CandEV { int eb, vb, e0, e1, v; };
struct CandEE { int b0, b1, a0, a1, c0, c1; };
struct CandFV { int fb, vb, f, v; };
struct Candidates {
    std::vector<CandVV> vv; std::vector<CandEV> ev; std::vector<CandEE> ee; std::vector<CandFV> fv;
    void clear() { vv.clear(); ev.clear(); ee.clear(); fv.clear(); }
};

}  // namespace

struct nxo_world {
    std::vector<Body> bodies;
    std::vector<Mesh> meshes;
    std::vector<Joint> joints;
    std::vector<Drive> drives;
    nxd_settings s;

    // IPCSolver state
    double kappa = 0.0, dhat = 1e-3, kappa_min = 0.0;
    bool barrier_initialized = false;   // the reference's process-static flag, per world
    std::vector<BodyContactMesh> bcm;
    Candidates cand;

    // forms installed for the Newton solve
    std::vector<Contact> barrier_contacts, friction_contacts;
    std::vector<double> normal_forces;
    bool barrier_form = false, friction_form = false, barrier_in_forms = false;
    double barrier_dhat = 1e-3, barrier_kappa = 0.0, friction_mu = 0.0, friction_eps = 1e-8, friction_dt = 0.01;
    // IPCSolver::allowed_contact_pair_keys_ / pair_friction_overrides_ (by body id)
    std::unordered_set<std::uint64_t> allowed_pairs;
    std::unordered_map<std::uint64_t, double> pair_friction;
    bool pair_allowed(int id_a, int id_b) const {
        if (allowed_pairs.empty()) return true;
        return allowed_pairs.count(pair_key(id_a, id_b)) != 0;
    }
    static std::uint64_t pair_key(int a, int b) {   // IPCSolver::makePairKey (IPCSolver.cpp:268-273)
        const int lo = std::min(a, b), hi = std::max(a, b);
        return ((std::uint64_t)(std::uint32_t)lo << 32) | (std::uint32_t)hi;
    }
    std::vector<double> x_hat;
    double dt = 0.01;               // integrator dt
    std::vector<double> x_prev, v_prev, a_prev;

    // diagnostics
    nxd_diagnostics diag{};
    double times[6] = {0, 0, 0, 0, 0, 0};

    // options
    int literal_min_distance = 1, md_stride = 1, num_threads = 1;
};

namespace {

inline V3 getv(const double* p, int i) { return mk(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
inline void setv(double* p, int i, V3 v) { p[3 * i] = v.x; p[3 * i + 1] = v.y; p[3 * i + 2] = v.z; }
inline V3 xseg(const std::vector<double>& x, int i) { return mk(x[i], x[i + 1], x[i + 2]); }

// Pairwise sum in a fixed tree: pad to a power of two with zeros, then
// v[i] += v[i + h] for h = P/2, P/4, ..., 1.  The reference's own order is
// not pinned (Eigen vectorises these reductions); this fixed order is the one
// the device reductions use, so both sides round identically.
double tree_sum(std::vector<double> v) {
    size_t P = 1;
    while (P < v.size()) P <<= 1;
    v.resize(P, 0.0);
    for (size_t h = P / 2; h >= 1; h /= 2) {
        for (size_t i = 0; i < h; ++i) v[i] = v[i] + v[i + h];
        if (h == 1) break;
    }
    return P ? v[0] : 0.0;
}

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// build_unique_edges (src/Physics/Contact/ContactAssembler.cpp:90-120): first-seen
// order over (v0,v1),(v1,v2),(v2,v0) of each face, stored as (min,max).
std::vector<std::array<int, 2>> build_unique_edges(const std::vector<std::array<int, 3>>& F) {
    std::unordered_set<std::uint64_t> seen;
    std::vector<std::array<int, 2>> E;
    E.reserve(F.size() * 3);
    for (const auto& f : F) {
        const std::array<std::pair<int, int>, 3> te = {std::make_pair(f[0], f[1]), std::make_pair(f[1], f[2]), std::make_pair(f[2], f[0])};
        for (const auto& [a, b] : te) {
            const int lo = std::min(a, b), hi = std::max(a, b);
            const std::uint64_t key = ((std::uint64_t)(std::uint32_t)lo << 32) | (std::uint32_t)hi;
            if (seen.insert(key).second) E.push_back({lo, hi});
        }
    }
    return E;
}

// transform_local_aabb (ContactAssembler.cpp:22-43)
AABB transform_local_aabb(V3 mn, V3 mx, V3 pos, Q q) {
    AABB box;
    for (int ix = 0; ix < 2; ++ix)
        for (int iy = 0; iy < 2; ++iy)
            for (int iz = 0; iz < 2; ++iz) {
                V3 c = mk(ix ? mx.x : mn.x, iy ? mx.y : mn.y, iz ? mx.z : mn.z);
                box.expand(pos + qrot(q, c));
            }
    return box;
}

// aabb_distance (ContactAssembler.cpp:45-55)
double aabb_distance(const AABB& a, const AABB& b) {
    const double dx = std::max({0.0, a.mn.x - b.mx.x, b.mn.x - a.mx.x});
    const double dy = std::max({0.0, a.mn.y - b.mx.y, b.mn.y - a.mx.y});
    const double dz = std::max({0.0, a.mn.z - b.mx.z, b.mn.z - a.mx.z});
    return std::sqrt(dx * dx + dy * dy + dz * dz);
}
// point_aabb_distance (ContactAssembler.cpp:57-65)
double point_aabb_distance(V3 p, const AABB& box) {
    const double dx = std::max({box.mn.x - p.x, 0.0, p.x - box.mx.x});
    const double dy = std::max({box.mn.y - p.y, 0.0, p.y - box.mx.y});
    const double dz = std::max({box.mn.z - p.z, 0.0, p.z - box.mx.z});
    return std::sqrt(dx * dx + dy * dy + dz * dz);
}

// select_top_k_indices (ContactAssembler.cpp:67-88)
std::vector<int> select_top_k_indices(int total, int k, const std::function<double(int)>& score) {
    if (total <= 0 || k <= 0) return {};
    std::vector<int> idx(total);
    std::iota(idx.begin(), idx.end(), 0);
    if (k < total) {
        std::nth_element(idx.begin(), idx.begin() + k, idx.end(), [&](int a, int b) { return score(a) < score(b); });
        idx.resize(k);
    }
    std::sort(idx.begin(), idx.end(), [&](int a, int b) { return score(a) < score(b); });
    return idx;
}

// ---------------------------------------------------------------------------
// ContactAssembler (src/Physics/Contact/ContactAssembler.cpp:124-343)
// ---------------------------------------------------------------------------
void assembler_build(nxo_world* w) {
    w->bcm.clear();
    w->bcm.reserve(w->bodies.size());
    for (size_t i = 0; i < w->bodies.size(); ++i) {
        const Body& b = w->bodies[i];
        if (b.mesh < 0) continue;
        BodyContactMesh m;
        m.body_id = b.id;
        m.world_index = (int)i;
        m.mesh = &w->meshes[b.mesh];
        m.world_position = b.position;
        m.world_orientation = b.orientation;
        m.world_aabb = transform_local_aabb(m.mesh->aabb_min, m.mesh->aabb_max, b.position, b.orientation);
        w->bcm.push_back(m);
    }
}

std::vector<std::pair<int, int>> detect_body_pairs(nxo_world* w, double r) {
    std::vector<std::pair<int, int>> out;
    if (w->bcm.size() < 2) return out;
    std::vector<AABB> aabbs;
    aabbs.reserve(w->bcm.size());
    for (const auto& m : w->bcm) aabbs.push_back(m.world_aabb.inflated(std::max(0.0, r)));
    // IncrementalBVHBroadPhase::detect after markNeedsRebuild (BroadPhase.cpp:84-131)
    BVH bvh;
    bvh.init(aabbs);
    std::vector<unsigned> ov;
    for (size_t i = 0; i < aabbs.size(); ++i) {
        bvh.intersectBox(aabbs[i], ov);
        for (unsigned j : ov)
            if ((size_t)j > i) out.emplace_back(w->bcm[i].world_index, w->bcm[j].world_index);
    }
    return out;
}

double estimate_min_body_pair_distance(nxo_world* w, double r) {
    if (w->bcm.size() < 2) return kInf;
    const auto pairs = detect_body_pairs(w, r);
    if (pairs.empty()) return kInf;
    double md = kInf;
    for (const auto& p : pairs) {
        int ia = -1, ib = -1;
        for (int k = 0; k < (int)w->bcm.size(); ++k) {
            if (w->bcm[k].world_index == p.first) ia = k;
            if (w->bcm[k].world_index == p.second) ib = k;
        }
        if (ia < 0 || ib < 0) continue;
        md = std::min(md, aabb_distance(w->bcm[ia].world_aabb, w->bcm[ib].world_aabb));
    }
    return md;
}

void candidates_for_pair(const BodyContactMesh* A, const BodyContactMesh* B, Candidates& out) {
    constexpr int kMax = 32;
    auto wv = [](const BodyContactMesh* m, int v) { return m->world_position + qrot(m->world_orientation, m->mesh->V[v]); };
    const Mesh& MA = *A->mesh; const Mesh& MB = *B->mesh;
    const int nVA = (int)MA.V.size(), nVB = (int)MB.V.size();
    const int nEA = (int)MA.E.size(), nEB = (int)MB.E.size();
    const int nFA = (int)MA.F.size(), nFB = (int)MB.F.size();
    const auto vA = select_top_k_indices(nVA, std::min(kMax, nVA), [&](int v) { return point_aabb_distance(wv(A, v), B->world_aabb); });
    const auto vB = select_top_k_indices(nVB, std::min(kMax, nVB), [&](int v) { return point_aabb_distance(wv(B, v), A->world_aabb); });
    const auto eA = select_top_k_indices(nEA, std::min(kMax, nEA), [&](int e) {
        return std::min(point_aabb_distance(wv(A, MA.E[e][0]), B->world_aabb), point_aabb_distance(wv(A, MA.E[e][1]), B->world_aabb)); });
    const auto eB = select_top_k_indices(nEB, std::min(kMax, nEB), [&](int e) {
        return std::min(point_aabb_distance(wv(B, MB.E[e][0]), A->world_aabb), point_aabb_distance(wv(B, MB.E[e][1]), A->world_aabb)); });
    const auto fA = select_top_k_indices(nFA, std::min(kMax, nFA), [&](int f) {
        return std::min({point_aabb_distance(wv(A, MA.F[f][0]), B->world_aabb), point_aabb_distance(wv(A, MA.F[f][1]), B->world_aabb),
                         point_aabb_distance(wv(A, MA.F[f][2]), B->world_aabb)}); });
    const auto fB = select_top_k_indices(nFB, std::min(kMax, nFB), [&](int f) {
        return std::min({point_aabb_distance(wv(B, MB.F[f][0]), A->world_aabb), point_aabb_distance(wv(B, MB.F[f][1]), A->world_aabb),
                         point_aabb_distance(wv(B, MB.F[f][2]), A->world_aabb)}); });
    for (int i : vA) for (int j : vB) out.vv.push_back({A->body_id, B->body_id, i, j});
    for (int i : eA) for (int j : vB) out.ev.push_back({A->body_id, B->body_id, MA.E[i][0], MA.E[i][1], j});
    for (int i : eB) for (int j : vA) out.ev.push_back({B->body_id, A->body_id, MB.E[i][0], MB.E[i][1], j});
    for (int i : eA) for (int j : eB) out.ee.push_back({A->body_id, B->body_id, MA.E[i][0], MA.E[i][1], MB.E[j][0], MB.E[j][1]});
    for (int i : fA) for (int j : vB) out.fv.push_back({A->body_id, B->body_id, i, j});
    for (int i : fB) for (int j : vA) out.fv.push_back({B->body_id, A->body_id, i, j});
}

void build_candidate_set(nxo_world* w, double act, Candidates& out) {
    out.clear();
    if (w->bcm.size() < 2) return;
    const auto pairs = detect_body_pairs(w, act);
    auto find_mesh = [&](int wi) -> const BodyContactMesh* {
        for (const auto& m : w->bcm) if (m.world_index == wi) return &m;
        return nullptr;
    };
    std::vector<std::pair<const BodyContactMesh*, const BodyContactMesh*>> work;
    for (const auto& p : pairs) {
        const BodyContactMesh* A = find_mesh(p.first);
        const BodyContactMesh* B = find_mesh(p.second);
        if (!A || !B) continue;
        if (aabb_distance(A->world_aabb, B->world_aabb) > act) continue;
        work.emplace_back(A, B);
    }
    w->diag.n_body_pairs = (int)work.size();
    if (w->num_threads <= 1 || work.size() < 2) {
        for (auto& ab : work) candidates_for_pair(ab.first, ab.second, out);
        return;
    }
    std::vector<Candidates> part(work.size());
#pragma omp parallel for schedule(dynamic, 1) num_threads(w->num_threads)
    for (long i = 0; i < (long)work.size(); ++i) candidates_for_pair(work[i].first, work[i].second, part[i]);
    for (auto& c : part) {
        out.vv.insert(out.vv.end(), c.vv.begin(), c.vv.end());
        out.ev.insert(out.ev.end(), c.ev.begin(), c.ev.end());
        out.ee.insert(out.ee.end(), c.ee.begin(), c.ee.end());
        out.fv.insert(out.fv.end(), c.fv.begin(), c.fv.end());
    }
}

// ---------------------------------------------------------------------------
// Barrier (src/Physics/Contact/Barrier.cpp:11-46)
// ---------------------------------------------------------------------------
double barrier_value(double d, double dh, double k) {
    if (d >= dh) return 0.0;
    if (d <= 0.0) return kInf;
    double r = d / dh;
    return -k * (d - dh) * (d - dh) * nxm::log(r);
}
double barrier_gradient(double d, double dh, double k) {
    if (d >= dh) return 0.0;
    if (d <= 0.0) return -kInf;
    double diff = d - dh;
    double lr = nxm::log(d / dh);
    return -k * (2 * diff * lr + diff * diff / d);
}
double barrier_hessian(double d, double dh, double k) {
    if (d >= dh) return 0.0;
    if (d <= 0.0) return kInf;
    double diff = d - dh;
    double lr = nxm::log(d / dh);
    return -k * (2 * lr + 4 * diff / d - (diff * diff) / (d * d));
}

// computeMinDistance (NexDynIPC/Physics/Contact/AdaptiveBarrier.h:89-128) for one
// vertex against one face, returning +inf when the barycentric test fails.
inline double vertex_face_plane_distance(V3 p, V3 v0, V3 v1, V3 v2) {
    V3 e1 = v1 - v0, e2 = v2 - v0;
    V3 n = cross(e1, e2);
    double area = norm(n);
    if (area < 1e-12) return kInf;
    n = normalized(n);
    double dist = std::fabs(dot(p - v0, n));
    // M = [e1 e2 n] (columns); coeffs = M^-1 (p - v0) by the cofactor inverse.
    double M[3][3] = {{e1.x, e2.x, n.x}, {e1.y, e2.y, n.y}, {e1.z, e2.z, n.z}};
    auto cof = [&](int i, int j) {
        const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
        return M[i1][j1] * M[i2][j2] - M[i1][j2] * M[i2][j1];
    };
    const double c00 = cof(0, 0), c10 = cof(1, 0), c20 = cof(2, 0);
    const double det = c00 * M[0][0] + c10 * M[1][0] + c20 * M[2][0];
    const double invdet = 1.0 / det;
    double inv[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) inv[i][j] = cof(j, i) * invdet;
    V3 r = p - v0;
    const double c0 = inv[0][0] * r.x + inv[0][1] * r.y + inv[0][2] * r.z;
    const double c1 = inv[1][0] * r.x + inv[1][1] * r.y + inv[1][2] * r.z;
    const double b0 = 1.0 - c0 - c1, b1 = c0, b2 = c1;
    const double bmin = std::min(std::min(b0, b1), b2), bmax = std::max(std::max(b0, b1), b2);
    if (bmin >= -1e-6 && bmax <= 1.0 + 1e-6) return dist;
    return kInf;
}

// computeSceneMinDistance (AdaptiveBarrier.h:130-162), literal loop nest.
double scene_min_distance_literal(nxo_world* w) {
    const int N = (int)w->bodies.size();
    double md = kInf;
    const int stride = std::max(1, w->md_stride);
#pragma omp parallel for schedule(dynamic, 1) reduction(min : md) num_threads(std::max(1, w->num_threads))
    for (int i = 0; i < N; ++i) {
        if (i % stride) continue;
        const Body& bi = w->bodies[i];
        if (bi.mesh < 0) continue;
        const Mesh& MA = w->meshes[bi.mesh];
        std::vector<V3> VBw;
        for (size_t vi = 0; vi < MA.V.size(); ++vi) {
            const V3 wvx = bi.position + qrot(bi.orientation, MA.V[vi]);
            for (int j = i + 1; j < N; ++j) {
                const Body& bj = w->bodies[j];
                if (bj.mesh < 0) continue;
                const Mesh& MB = w->meshes[bj.mesh];
                VBw.resize(MB.V.size());
                for (size_t k = 0; k < MB.V.size(); ++k) VBw[k] = bj.position + qrot(bj.orientation, MB.V[k]);
                double d = kInf;
                for (const auto& f : MB.F) d = std::min(d, vertex_face_plane_distance(wvx, VBw[f[0]], VBw[f[1]], VBw[f[2]]));
                md = std::min(md, d);
            }
        }
    }
    return md;
}

// Pruned form of the same loop nest.  A (vertex p of body i, face of body j)
// test that passes the barycentric check with plane distance d puts p within
// d + tol_j of body j's world AABB, tol_j covering the 1e-6 barycentric slack
// times the face size plus rounding.  Tests whose vertex lies farther than
// kPruneBand + tol_j from that AABB therefore cannot produce a distance below
// kPruneBand, and the minimum is unchanged whenever it is below kPruneBand.
constexpr double kPruneBand = 1e-6;
double scene_min_distance_pruned(nxo_world* w) {
    const int N = (int)w->bodies.size();
    std::vector<AABB> box(N);
    std::vector<double> tol(N, 0.0);
    std::vector<std::vector<V3>> WV(N);
    for (int j = 0; j < N; ++j) {
        const Body& b = w->bodies[j];
        if (b.mesh < 0) continue;
        const Mesh& M = w->meshes[b.mesh];
        box[j] = transform_local_aabb(M.aabb_min, M.aabb_max, b.position, b.orientation);
        WV[j].resize(M.V.size());
        for (size_t k = 0; k < M.V.size(); ++k) WV[j][k] = b.position + qrot(b.orientation, M.V[k]);
        const double diag = norm(M.aabb_max - M.aabb_min);
        tol[j] = 4e-6 * diag + 1e-9 * (1.0 + norm(b.position) + diag);
    }
    double md = kInf;
#pragma omp parallel for schedule(dynamic, 1) reduction(min : md) num_threads(std::max(1, w->num_threads))
    for (int i = 0; i < N; ++i) {
        const Body& bi = w->bodies[i];
        if (bi.mesh < 0) continue;
        for (int j = i + 1; j < N; ++j) {
            const Body& bj = w->bodies[j];
            if (bj.mesh < 0) continue;
            const double band = kPruneBand + tol[j];
            if (aabb_distance(box[i], box[j]) > band) continue;
            const Mesh& MB = w->meshes[bj.mesh];
            for (const V3& p : WV[i]) {
                if (point_aabb_distance(p, box[j]) > band) continue;
                for (const auto& f : MB.F) {
                    const V3 a = WV[j][f[0]], b = WV[j][f[1]], c = WV[j][f[2]];
                    AABB fb; fb.expand(a); fb.expand(b); fb.expand(c);
                    if (point_aabb_distance(p, fb) > band) continue;
                    md = std::min(md, vertex_face_plane_distance(p, a, b, c));
                }
            }
        }
    }
    return md;
}

// ---------------------------------------------------------------------------
// CCD (NexDynIPC/Physics/Contact/CCD/*.h, src/Physics/Contact/CCD/TimeOfImpact.cpp)
// ---------------------------------------------------------------------------
struct Ivl { double lo, hi; };
inline Ivl iv(double a) { return {a, a}; }
inline Ivl iv(double a, double b) { return {a, b}; }
inline double dn(double v) { return std::nextafter(v, -kInf); }
inline double up(double v) { return std::nextafter(v, kInf); }
inline Ivl operator+(Ivl a, Ivl b) { return {dn(a.lo + b.lo), up(a.hi + b.hi)}; }
inline Ivl operator-(Ivl a, Ivl b) { return {dn(a.lo - b.hi), up(a.hi - b.lo)}; }
inline Ivl operator*(Ivl a, Ivl b) {
    const double p[4] = {a.lo * b.lo, a.lo * b.hi, a.hi * b.lo, a.hi * b.hi};
    return {dn(*std::min_element(p, p + 4)), up(*std::max_element(p, p + 4))};
}
inline bool zero_in(Ivl a) { return a.lo <= 0.0 && 0.0 <= a.hi; }
struct V3I { Ivl x, y, z; };

// Quaternion slerp as Eigen's QuaternionBase::slerp (linear when |dot| ~ 1).
Q slerp(Q a, double t, Q b) {
    const double one = 1.0 - std::numeric_limits<double>::epsilon();
    const double d = a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w;
    const double ad = std::fabs(d);
    double s0, s1;
    if (ad >= one) { s0 = 1.0 - t; s1 = t; }
    else {
        const double th = std::acos(ad), st = std::sin(th);
        s0 = std::sin((1.0 - t) * th) / st; s1 = std::sin(t * th) / st;
    }
    if (d < 0) s1 = -s1;
    return mkq(s0 * a.w + s1 * b.w, s0 * a.x + s1 * b.x, s0 * a.y + s1 * b.y, s0 * a.z + s1 * b.z);
}
// vertexTrajectoryAABB (RigidTrajectoryAABB.h:57-72)
V3I vertex_traj(V3I pos, Q q0, Q q1, Ivl t, V3 lp) {
    Q ql = slerp(q0, t.lo, q1), qh = slerp(q0, t.hi, q1);
    V3 pl = qrot(ql, lp), ph = qrot(qh, lp);
    V3I r{iv(std::min(pl.x, ph.x), std::max(pl.x, ph.x)), iv(std::min(pl.y, ph.y), std::max(pl.y, ph.y)),
          iv(std::min(pl.z, ph.z), std::max(pl.z, ph.z))};
    return {pos.x + r.x, pos.y + r.y, pos.z + r.z};
}

// computeFaceVertexTOIImpl (TimeOfImpact.cpp:97-150) with intervalRootFinderImpl
// (IntervalRootFinder.h:20-114).  The probe f(x_tol) is evaluated as the
// reference does; the root box x0 = ([0,toi],[0,1],[0,1]) is then tested by the
// domain predicate, whose w = 1-u-v = [-1,1] fails lower(w) >= 0, so the box is
// discarded before any bisection and the call reports no impact.
bool face_vertex_toi(const Body& vb, V3 vp0, Q vq0, V3 vp1, Q vq1, V3 lv, const Body& fb, V3 fp0, Q fq0, V3 fp1, Q fq1,
                     V3 f0, V3 f1, V3 f2, double& toi, double earliest, double tol0) {
    (void)vb; (void)fb;
    V3I pv{iv(std::min(vp0.x, vp1.x), std::max(vp0.x, vp1.x)), iv(std::min(vp0.y, vp1.y), std::max(vp0.y, vp1.y)),
           iv(std::min(vp0.z, vp1.z), std::max(vp0.z, vp1.z))};
    V3I pf{iv(std::min(fp0.x, fp1.x), std::max(fp0.x, fp1.x)), iv(std::min(fp0.y, fp1.y), std::max(fp0.y, fp1.y)),
           iv(std::min(fp0.z, fp1.z), std::max(fp0.z, fp1.z))};
    auto f = [&](Ivl t, Ivl u, Ivl v) {
        V3I a = vertex_traj(pv, vq0, vq1, t, lv);
        V3I w0 = vertex_traj(pf, fq0, fq1, t, f0), w1 = vertex_traj(pf, fq0, fq1, t, f1), w2 = vertex_traj(pf, fq0, fq1, t, f2);
        Ivl wi = (iv(1.0) - u) - v;
        V3I fpnt{wi * w0.x + u * w1.x + v * w2.x, wi * w0.y + u * w1.y + v * w2.y, wi * w0.z + u * w1.z + v * w2.z};
        return V3I{a.x - fpnt.x, a.y - fpnt.y, a.z - fpnt.z};
    };
    // probe at x_tol (its only effect is a tolerance that the search never reads)
    V3I probe = f(iv(0, tol0), iv(0, 1), iv(0, 1));
    volatile bool zi = zero_in(probe.x) && zero_in(probe.y) && zero_in(probe.z);
    (void)zi;
    // stack search: the initial box fails the domain predicate
    const Ivl u = iv(0, 1), v = iv(0, 1);
    const Ivl wv = (iv(1.0) - u) - v;
    const bool valid = u.lo >= 0 && u.hi <= 1 && v.lo >= 0 && v.hi <= 1 && wv.lo >= 0 && wv.hi <= 1;
    (void)earliest;
    if (!valid) { toi = kInf; return false; }
    // A valid domain would continue with bisection; unreachable for this predicate.
    toi = kInf;
    return false;
}

double compute_earliest_toi(nxo_world* w, double dt) {
    if (w->bodies.empty() || w->cand.fv.empty()) return 1.0;
    std::unordered_map<int, int> id2i;
    for (int i = 0; i < (int)w->bodies.size(); ++i) id2i[w->bodies[i].id] = i;
    double earliest = 1.0;
    const long nfv = (long)w->cand.fv.size();
    std::vector<double> tois(nfv, kInf);
    std::vector<char> hit(nfv, 0);
#pragma omp parallel for schedule(static) num_threads(std::max(1, w->num_threads))
    for (long c = 0; c < nfv; ++c) {
        const CandFV& fv = w->cand.fv[c];
        auto itf = id2i.find(fv.fb), itv = id2i.find(fv.vb);
        if (itf == id2i.end() || itv == id2i.end()) continue;
        const Body& fb = w->bodies[itf->second];
        const Body& vb = w->bodies[itv->second];
        if (fb.mesh < 0 || vb.mesh < 0) continue;
        const Mesh& FM = w->meshes[fb.mesh];
        const Mesh& VM = w->meshes[vb.mesh];
        V3 fp1 = fb.position + fb.velocity * dt, vp1 = vb.position + vb.velocity * dt;
        double toi = kInf;
        hit[c] = face_vertex_toi(vb, vb.position, vb.orientation, vp1, vb.orientation, VM.V[fv.v], fb, fb.position, fb.orientation,
                                 fp1, fb.orientation, FM.V[FM.F[fv.f][0]], FM.V[FM.F[fv.f][1]], FM.V[FM.F[fv.f][2]], toi,
                                 earliest, 1e-8);
        tois[c] = toi;
    }
    for (long c = 0; c < nfv; ++c)
        if (hit[c] && tois[c] < earliest) earliest = tois[c];
    return earliest;
}

// IPCSolver::computeMaxStep (IPCSolver.cpp:355-392)
double compute_max_step(nxo_world* w, double dt) {
    if (!w->s.enable_ccd || w->bodies.empty()) return dt;
    double max_speed = 0.0;
    for (const auto& b : w->bodies) max_speed = std::max(max_speed, norm(b.velocity));
    const double infl = std::max(1e-6, w->dhat) + max_speed * dt;
    const auto close = detect_body_pairs(w, infl);
    // no allowed-pair list: every pair is allowed (IPCSolver.cpp:283-289)
    if (close.empty()) return dt;
    if (w->cand.fv.empty()) return dt;
    const double toi = compute_earliest_toi(w, dt);
    if (toi < 1.0) return toi * w->s.ccd_safety_factor * dt;
    return dt;
}

// ---------------------------------------------------------------------------
// Contact detection (IPCSolver.cpp:32-134 helpers, 394-806)
// ---------------------------------------------------------------------------
void closest_points_on_segments(V3 p1, V3 q1, V3 p2, V3 q2, V3& c1, V3& c2) {
    constexpr double eps = 1e-12;
    const V3 d1 = q1 - p1, d2 = q2 - p2, r = p1 - p2;
    const double a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
    double s, t;
    if (a <= eps && e <= eps) { c1 = p1; c2 = p2; return; }
    if (a <= eps) {
        s = 0.0; t = std::clamp(f / e, 0.0, 1.0);
    } else {
        const double c = dot(d1, r);
        if (e <= eps) {
            t = 0.0; s = std::clamp(-c / a, 0.0, 1.0);
        } else {
            const double b = dot(d1, d2);
            const double denom = a * e - b * b;
            if (std::fabs(denom) > eps) s = std::clamp((b * f - c * e) / denom, 0.0, 1.0);
            else s = 0.0;
            t = (b * s + f) / e;
            if (t < 0.0) { t = 0.0; s = std::clamp(-c / a, 0.0, 1.0); }
            else if (t > 1.0) { t = 1.0; s = std::clamp((b - c) / a, 0.0, 1.0); }
        }
    }
    c1 = p1 + d1 * s;
    c2 = p2 + d2 * t;
}
V3 safe_normalized(V3 v, V3 fb) {
    const double n = norm(v);
    if (n > 1e-12) return v / n;
    const double fn = norm(fb);
    if (fn > 1e-12) return fb / fn;
    return mk(0, 1, 0);
}
bool point_in_triangle(V3 p, V3 a, V3 b, V3 c, double eps = 1e-8) {
    const V3 v0 = b - a, v1 = c - a, v2 = p - a;
    const double d00 = dot(v0, v0), d01 = dot(v0, v1), d11 = dot(v1, v1), d20 = dot(v2, v0), d21 = dot(v2, v1);
    const double denom = d00 * d11 - d01 * d01;
    if (std::fabs(denom) < 1e-16) return false;
    const double v = (d11 * d20 - d01 * d21) / denom;
    const double ww = (d00 * d21 - d01 * d20) / denom;
    const double u = 1.0 - v - ww;
    return u >= -eps && v >= -eps && ww >= -eps;
}

struct PoseFn {
    // per world index: position and orientation used for the contact test
    std::vector<V3> p; std::vector<Q> q;
};

// One detection pass.  With x == nullptr the poses are the bodies' current
// ones (detectContacts); otherwise p = x[6i..], q = exp(theta) q_body with the
// '>' threshold (detectContactsAtState).
std::vector<Contact> detect_contacts(nxo_world* w, const std::vector<double>* x, int* raw_count) {
    std::vector<Contact> contacts;
    if (raw_count) *raw_count = 0;
    if (w->bodies.empty()) return contacts;
    std::unordered_map<int, int> id2i;
    id2i.reserve(w->bodies.size());
    for (int i = 0; i < (int)w->bodies.size(); ++i) id2i[w->bodies[i].id] = i;
    std::unordered_map<int, const BodyContactMesh*> id2m;
    for (const auto& m : w->bcm) id2m[m.body_id] = &m;
    const double dh = w->dhat;
    constexpr size_t kMaxRaw = 40000, kMax = 2000;

    auto pose = [&](int wi, V3& p, Q& q) {
        if (!x) { p = w->bodies[wi].position; q = w->bodies[wi].orientation; return; }
        const int d = wi * 6;
        p = xseg(*x, d);
        q = update_rotation_gt(w->bodies[wi].orientation, xseg(*x, d + 3));
    };
    auto world_vertex = [&](int bid, int lv, V3& out) -> bool {
        auto mit = id2m.find(bid);
        auto bit = id2i.find(bid);
        if (mit == id2m.end() || bit == id2i.end()) return false;
        const Mesh* M = mit->second->mesh;
        if (lv < 0 || lv >= (int)M->V.size()) return false;
        V3 p; Q q; pose(bit->second, p, q);
        out = p + qrot(q, M->V[lv]);
        return true;
    };
    struct Raw { int a, b, type, pa, pb; V3 point, normal; double dist; };
    auto finish = [&](const Raw& r, std::vector<Contact>& out) {
        auto ait = id2i.find(r.a), bit = id2i.find(r.b);
        if (ait == id2i.end() || bit == id2i.end()) return;
        if (!w->pair_allowed(r.a, r.b)) return;   // IPCSolver.cpp:448, 668
        V3 pa, pb; Q qa, qb;
        pose(ait->second, pa, qa); pose(bit->second, pb, qb);
        V3 n = safe_normalized(r.normal, pb - pa);
        if (dot(n, pb - pa) < 0.0) n = -n;
        Contact c;
        c.bodyA = ait->second; c.bodyB = bit->second; c.type = r.type; c.primA = r.pa; c.primB = r.pb;
        c.point = r.point; c.normal = n; c.distance = std::max(0.0, r.dist);
        out.push_back(c);
    };
    auto fv_test = [&](const CandFV& cd, std::vector<Contact>& out) {
        auto fit = id2m.find(cd.fb);
        if (fit == id2m.end()) return;
        const Mesh* FM = fit->second->mesh;
        if (cd.f < 0 || cd.f >= (int)FM->F.size()) return;
        V3 v0, v1, v2, p;
        if (!world_vertex(cd.fb, FM->F[cd.f][0], v0) || !world_vertex(cd.fb, FM->F[cd.f][1], v1) ||
            !world_vertex(cd.fb, FM->F[cd.f][2], v2) || !world_vertex(cd.vb, cd.v, p)) return;
        const V3 n = safe_normalized(cross(v1 - v0, v2 - v0), mk(0, 1, 0));
        const double sd = dot(p - v0, n);
        const double dist = std::fabs(sd);
        if (dist >= dh) return;
        const V3 proj = p - sd * n;
        if (!point_in_triangle(proj, v0, v1, v2)) return;
        finish({cd.fb, cd.vb, 0, cd.f, cd.v, 0.5 * (proj + p), (sd >= 0.0) ? n : -n, dist}, out);
    };
    auto ee_test = [&](const CandEE& cd, std::vector<Contact>& out) {
        V3 a0, a1, b0, b1;
        if (!world_vertex(cd.b0, cd.a0, a0) || !world_vertex(cd.b0, cd.a1, a1) || !world_vertex(cd.b1, cd.c0, b0) ||
            !world_vertex(cd.b1, cd.c1, b1)) return;
        V3 c0, c1;
        closest_points_on_segments(a0, a1, b0, b1, c0, c1);
        const V3 delta = c1 - c0;
        const double dist = norm(delta);
        if (dist >= dh) return;
        finish({cd.b0, cd.b1, 1, cd.a0, cd.c0, 0.5 * (c0 + c1), delta, dist}, out);
    };
    auto vv_test = [&](const CandVV& cd, std::vector<Contact>& out) {
        V3 a, b;
        if (!world_vertex(cd.b0, cd.v0, a) || !world_vertex(cd.b1, cd.v1, b)) return;
        const V3 d = b - a;
        const double dist = norm(d);
        if (dist >= dh) return;
        finish({cd.b0, cd.b1, 0, cd.v0, cd.v1, 0.5 * (a + b), d, dist}, out);
    };
    // The per-candidate tests are independent; run them in chunks and append
    // in candidate order, then apply the reference's raw cap in that order.
    auto run = [&](auto& list, auto&& test) {
        const long n = (long)list.size();
        if (w->num_threads <= 1 || n < 4096) {
            for (long i = 0; i < n && contacts.size() < kMaxRaw; ++i) test(list[i], contacts);
            return;
        }
        const long chunk = 4096;
        const long nch = (n + chunk - 1) / chunk;
        std::vector<std::vector<Contact>> part(nch);
#pragma omp parallel for schedule(dynamic, 1) num_threads(w->num_threads)
        for (long c = 0; c < nch; ++c)
            for (long i = c * chunk; i < std::min(n, (c + 1) * chunk); ++i) test(list[i], part[c]);
        for (auto& p : part)
            for (auto& c : p) { if (contacts.size() >= kMaxRaw) return; contacts.push_back(c); }
    };
    run(w->cand.fv, fv_test);
    run(w->cand.ee, ee_test);
    if (contacts.empty()) run(w->cand.vv, vv_test);
    if (raw_count) *raw_count = (int)contacts.size();
    if (contacts.size() > kMax) {
        std::sort(contacts.begin(), contacts.end(), [](const Contact& a, const Contact& b) { return a.distance < b.distance; });
        contacts.resize(kMax);
    }
    return contacts;
}

// ---------------------------------------------------------------------------
// Joints (src/Dynamics/Joints/*.cpp, NexDynIPC/Dynamics/Joints/JointPrimitives.h)
// ---------------------------------------------------------------------------
struct EvalBody { V3 p; Q q; };
inline EvalBody eval_body(int g, V3 p_ref, Q q_ref, const std::vector<double>& x) {
    EvalBody e;
    if (g >= 0) { e.p = xseg(x, g); e.q = update_rotation_joint(q_ref, xseg(x, g + 3)); }
    else { e.p = p_ref; e.q = q_ref; }
    return e;
}
inline M3 cross_mat(V3 v) {
    M3 M;
    M(0, 0) = 0.0; M(0, 1) = -v.z; M(0, 2) = v.y;
    M(1, 0) = v.z; M(1, 1) = 0.0; M(1, 2) = -v.x;
    M(2, 0) = -v.y; M(2, 1) = v.x; M(2, 2) = 0.0;
    return M;
}
inline M3 mat_mul(const M3& A, const M3& B) {
    M3 C;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) C(i, j) = A(i, 0) * B(0, j) + A(i, 1) * B(1, j) + A(i, 2) * B(2, j);
    return C;
}

// JointPrimitives::computeBasis (JointPrimitives.h:29-37)
void compute_basis(V3 axis, V3& u, V3& v) {
    const V3 a = normalized(axis);
    u = std::abs(a.x) < 0.8 ? normalized(cross(a, mk(1, 0, 0))) : normalized(cross(a, mk(0, 1, 0)));
    v = normalized(cross(a, u));
}

// C(x) per joint kind
void joint_C(const Joint& J, const std::vector<double>& x, double* C) {
    switch (J.type) {
        case NXD_JOINT_HINGE:
        case NXD_JOINT_SPHERICAL: {
            const EvalBody A = eval_body(J.gA, J.pA_ref, J.qA_ref, x);
            const EvalBody B = eval_body(J.gB, J.pB_ref, J.qB_ref, x);
            // PointPrimitive::value (JointPrimitives.h:52-56)
            const V3 rA = qrot(A.q, J.anchorA), rB = qrot(B.q, J.anchorB);
            const V3 v = (A.p + rA) - (B.p + rB);
            C[0] = v.x; C[1] = v.y; C[2] = v.z;
            if (J.type == NXD_JOINT_HINGE) {
                // AxisCrossPrimitive::value (JointPrimitives.h:206-210)
                const V3 c = cross(qrot(A.q, J.axisA), qrot(B.q, J.axisB));
                C[3] = c.x; C[4] = c.y; C[5] = c.z;
            }
            break;
        }
        case NXD_JOINT_FIXED: {
            // FixedJoint::computeC (FixedJoint.cpp:23-42)
            if (J.gA < 0) { for (int i = 0; i < 6; ++i) C[i] = 0; break; }
            const V3 p = xseg(x, J.gA);
            const V3 d = p - J.target_pos;
            C[0] = d.x; C[1] = d.y; C[2] = d.z;
            // FixedOrientationPrimitive::value (JointPrimitives.h:288-298)
            const Q dq = qmul(J.target_ori, qconj(J.qA_ref));
            double ang; V3 ax;
            q_to_angle_axis(dq, ang, ax);
            const V3 tt = ax * ang;
            const V3 th = xseg(x, J.gA + 3);
            C[3] = th.x - tt.x; C[4] = th.y - tt.y; C[5] = th.z - tt.z;
            break;
        }
        case NXD_JOINT_PRISMATIC:
        case NXD_JOINT_CYLINDRICAL: {
            const EvalBody A = eval_body(J.gA, J.pA_ref, J.qA_ref, x);
            const EvalBody B = eval_body(J.gB, J.pB_ref, J.qB_ref, x);
            // PointOnAxisPrimitive::value (JointPrimitives.h:117-124)
            const V3 rA = qrot(A.q, J.anchorA), rB = qrot(B.q, J.anchorB);
            const V3 d = (B.p + rB) - (A.p + rA);
            const V3 uAw = qrot(A.q, J.uA), vAw = qrot(A.q, J.vA);
            C[0] = dot(d, uAw); C[1] = dot(d, vAw);
            // DirectionPrimitive::value (JointPrimitives.h:170-175)
            const V3 nA = qrot(A.q, J.axisA), uBw = qrot(B.q, J.uB), vBw = qrot(B.q, J.vB);
            C[2] = dot(nA, uBw); C[3] = dot(nA, vBw);
            // RollLockPrimitive::value (JointPrimitives.h:245-249)
            if (J.type == NXD_JOINT_PRISMATIC) C[4] = dot(uAw, vBw);
            break;
        }
        case NXD_JOINT_DISTANCE_LIMIT: {
            // DistanceLimitJoint::computeC (DistanceLimitJoint.cpp:49-58)
            const V3 pA = J.gA >= 0 ? xseg(x, J.gA) : J.pA_ref, pB = J.gB >= 0 ? xseg(x, J.gB) : J.pB_ref;
            const double dist = norm(pB - pA);
            C[0] = J.min_dist - dist;
            C[1] = dist - J.max_dist;
            break;
        }
        case NXD_JOINT_ANGLE_LIMIT: {
            // AngleLimitJoint::currentRelativeAngle (AngleLimitJoint.cpp:45-63)
            Q qA = J.qA_ref, qB = J.qB_ref;
            if (J.gA >= 0 && J.gA + 5 < (int)x.size()) qA = update_rotation_joint(J.qA_ref, xseg(x, J.gA + 3));
            if (J.gB >= 0 && J.gB + 5 < (int)x.size()) qB = update_rotation_joint(J.qB_ref, xseg(x, J.gB + 3));
            const Q qr = qmul(qconj(qA), qB);
            double ang; V3 ax;
            q_to_angle_axis(qr, ang, ax);
            const double a = ang * dot(ax, J.axis);
            C[0] = J.min_angle - a;
            C[1] = a - J.max_angle;
            break;
        }
    }
}

// Jacobian as a small dense matrix over the joint's columns: cols[k] is a global
// DOF index; the reference builds the same entries as sparse triplets and sums
// duplicates (setFromTriplets).
struct JacRows {
    int dim = 0;
    std::vector<int> cols;               // sorted unique global columns
    std::vector<double> J;               // dim x cols.size()
    int col(int g) {
        for (size_t k = 0; k < cols.size(); ++k) if (cols[k] == g) return (int)k;
        return -1;
    }
};
void jac_add(std::vector<Trip>& t, int r, int c, double v) { t.push_back({r, c, v}); }
void point_rows(std::vector<Trip>& t, int row, int gA, int gB, V3 rA, V3 rB) {
    // PointPrimitive::addJacobianRows (JointPrimitives.h:58-90)
    if (gA >= 0) {
        jac_add(t, row + 0, gA + 0, 1.0); jac_add(t, row + 1, gA + 1, 1.0); jac_add(t, row + 2, gA + 2, 1.0);
        M3 dr = cross_mat(rA);
        for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) jac_add(t, row + i, gA + 3 + j, -dr(i, j));
    }
    if (gB >= 0) {
        jac_add(t, row + 0, gB + 0, -1.0); jac_add(t, row + 1, gB + 1, -1.0); jac_add(t, row + 2, gB + 2, -1.0);
        M3 dr = cross_mat(rB);
        for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) jac_add(t, row + i, gB + 3 + j, dr(i, j));
    }
}
JacRows joint_J(const Joint& J, const std::vector<double>& x) {
    std::vector<Trip> t;
    JacRows R;
    R.dim = J.dim();
    switch (J.type) {
        case NXD_JOINT_HINGE:
        case NXD_JOINT_SPHERICAL: {
            const EvalBody A = eval_body(J.gA, J.pA_ref, J.qA_ref, x);
            const EvalBody B = eval_body(J.gB, J.pB_ref, J.qB_ref, x);
            point_rows(t, 0, J.gA, J.gB, qrot(A.q, J.anchorA), qrot(B.q, J.anchorB));
            if (J.type == NXD_JOINT_HINGE) {
                // AxisCrossPrimitive::addJacobianRows (JointPrimitives.h:212-240)
                const V3 nA = qrot(A.q, J.axisA), nB = qrot(B.q, J.axisB);
                if (J.gA >= 0) {
                    M3 dA = mat_mul(cross_mat(nB), cross_mat(nA));
                    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) jac_add(t, 3 + i, J.gA + 3 + j, dA(i, j));
                }
                if (J.gB >= 0) {
                    M3 ma = cross_mat(nA);
                    for (int k = 0; k < 9; ++k) ma.m[k] = -ma.m[k];
                    M3 dB = mat_mul(ma, cross_mat(nB));
                    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) jac_add(t, 3 + i, J.gB + 3 + j, dB(i, j));
                }
            }
            break;
        }
        case NXD_JOINT_FIXED: {
            // FixedPositionPrimitive / FixedOrientationPrimitive rows (JointPrimitives.h:267-313)
            if (J.gA >= 0) {
                for (int i = 0; i < 3; ++i) jac_add(t, i, J.gA + i, 1.0);
                for (int i = 0; i < 3; ++i) jac_add(t, 3 + i, J.gA + 3 + i, 1.0);
            }
            break;
        }
        case NXD_JOINT_PRISMATIC:
        case NXD_JOINT_CYLINDRICAL: {
            const EvalBody A = eval_body(J.gA, J.pA_ref, J.qA_ref, x);
            const EvalBody B = eval_body(J.gB, J.pB_ref, J.qB_ref, x);
            const V3 rA = qrot(A.q, J.anchorA), rB = qrot(B.q, J.anchorB);
            const V3 d = (B.p + rB) - (A.p + rA);
            const V3 uAw = qrot(A.q, J.uA), vAw = qrot(A.q, J.vA);
            // PointOnAxisPrimitive::addJacobianRows (JointPrimitives.h:126-163)
            const V3 dirs[2] = {uAw, vAw};
            for (int r = 0; r < 2; ++r) {
                const V3 dir = dirs[r];
                if (J.gA >= 0) {
                    for (int k = 0; k < 3; ++k) jac_add(t, r, J.gA + k, -dir[k]);
                    const V3 gA = cross(dir, rA) + cross(dir, d);
                    for (int k = 0; k < 3; ++k) jac_add(t, r, J.gA + 3 + k, gA[k]);
                }
                if (J.gB >= 0) {
                    for (int k = 0; k < 3; ++k) jac_add(t, r, J.gB + k, dir[k]);
                    const V3 gB = cross(rB, dir);
                    for (int k = 0; k < 3; ++k) jac_add(t, r, J.gB + 3 + k, gB[k]);
                }
            }
            // DirectionPrimitive::addJacobianRows (JointPrimitives.h:177-200)
            const V3 nA = qrot(A.q, J.axisA), uBw = qrot(B.q, J.uB), vBw = qrot(B.q, J.vB);
            const V3 bdirs[2] = {uBw, vBw};
            for (int r = 0; r < 2; ++r) {
                if (J.gA >= 0) { const V3 gA = cross(nA, bdirs[r]); for (int k = 0; k < 3; ++k) jac_add(t, 2 + r, J.gA + 3 + k, gA[k]); }
                if (J.gB >= 0) { const V3 gB = cross(bdirs[r], nA); for (int k = 0; k < 3; ++k) jac_add(t, 2 + r, J.gB + 3 + k, gB[k]); }
            }
            // RollLockPrimitive::addJacobianRow (JointPrimitives.h:251-265)
            if (J.type == NXD_JOINT_PRISMATIC) {
                if (J.gA >= 0) { const V3 gA = cross(uAw, vBw); for (int k = 0; k < 3; ++k) jac_add(t, 4, J.gA + 3 + k, gA[k]); }
                if (J.gB >= 0) { const V3 gB = cross(vBw, uAw); for (int k = 0; k < 3; ++k) jac_add(t, 4, J.gB + 3 + k, gB[k]); }
            }
            break;
        }
        case NXD_JOINT_DISTANCE_LIMIT: {
            // DistanceLimitJoint::direction / computeJ (DistanceLimitJoint.cpp:37-47, 60-89)
            const V3 pA = J.gA >= 0 ? xseg(x, J.gA) : J.pA_ref, pB = J.gB >= 0 ? xseg(x, J.gB) : J.pB_ref;
            const V3 dd = pB - pA;
            const double dist = norm(dd);
            const V3 dir = dist < 1e-12 ? mk(1, 0, 0) : dd / dist;
            if (J.gA >= 0) for (int k = 0; k < 3; ++k) { jac_add(t, 0, J.gA + k, dir[k]); jac_add(t, 1, J.gA + k, -dir[k]); }
            if (J.gB >= 0) for (int k = 0; k < 3; ++k) { jac_add(t, 0, J.gB + k, -dir[k]); jac_add(t, 1, J.gB + k, dir[k]); }
            break;
        }
        case NXD_JOINT_ANGLE_LIMIT: {
            // AngleLimitJoint::computeJ (AngleLimitJoint.cpp:74-96)
            if (J.gA >= 0) for (int k = 0; k < 3; ++k) { jac_add(t, 0, J.gA + 3 + k, J.axis[k]); jac_add(t, 1, J.gA + 3 + k, -J.axis[k]); }
            if (J.gB >= 0) for (int k = 0; k < 3; ++k) { jac_add(t, 0, J.gB + 3 + k, -J.axis[k]); jac_add(t, 1, J.gB + 3 + k, J.axis[k]); }
            break;
        }
    }
    for (const auto& tr : t) R.cols.push_back(tr.c);
    std::sort(R.cols.begin(), R.cols.end());
    R.cols.erase(std::unique(R.cols.begin(), R.cols.end()), R.cols.end());
    R.J.assign((size_t)R.dim * R.cols.size(), 0.0);
    for (const auto& tr : t) R.J[(size_t)tr.r * R.cols.size() + R.col(tr.c)] += tr.v;
    return R;
}

double joint_value(const Joint& J, const std::vector<double>& x) {
    double C[6];
    joint_C(J, x, C);
    const int d = J.dim();
    if (J.is_limit()) {
        // AngleLimitJoint::value (AngleLimitJoint.cpp:98-109), DistanceLimitJoint::value (:91-100)
        double e = 0.0;
        for (int i = 0; i < d; ++i) { const double gp = std::max(C[i], 0.0); e += J.lambda[i] * gp + 0.5 * J.mu * gp * gp; }
        return e;
    }
    // Joint::value (Joint.cpp:5-18)
    double t1 = 0.0, sq = 0.0;
    for (int i = 0; i < d; ++i) { t1 += J.lambda[i] * C[i]; sq += C[i] * C[i]; }
    return t1 + 0.5 * J.mu * sq;
}
void joint_gradient(const Joint& J, const std::vector<double>& x, std::vector<double>& g) {
    double C[6];
    joint_C(J, x, C);
    const int d = J.dim();
    double f[6];
    if (J.is_limit()) {
        for (int i = 0; i < d; ++i) f[i] = C[i] > 0.0 ? J.lambda[i] + J.mu * C[i] : 0.0;
    } else {
        for (int i = 0; i < d; ++i) f[i] = J.mu * C[i] + J.lambda[i];
    }
    JacRows R = joint_J(J, x);
    const size_t nc = R.cols.size();
    for (size_t k = 0; k < nc; ++k) {
        double s = 0.0;
        for (int r = 0; r < d; ++r) s += R.J[r * nc + k] * f[r];
        g[R.cols[k]] += s;
    }
}
void joint_hessian(const Joint& J, const std::vector<double>& x, std::vector<Trip>& t) {
    if (J.type == NXD_JOINT_ANGLE_LIMIT) {
        // AngleLimitJoint::hessian (AngleLimitJoint.cpp:127-168)
        double C[2];
        joint_C(J, x, C);
        const bool amin = C[0] > 0.0, amax = C[1] > 0.0;
        if (!amin && !amax) return;
        double H[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int rep = 0; rep < 2; ++rep) {
            if ((rep == 0 && amin) || (rep == 1 && amax))
                for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) H[i][j] += J.mu * (J.axis[i] * J.axis[j]);
        }
        if (J.gA >= 0) for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) t.push_back({J.gA + 3 + i, J.gA + 3 + j, H[i][j]});
        if (J.gB >= 0) for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) t.push_back({J.gB + 3 + i, J.gB + 3 + j, H[i][j]});
        if (J.gA >= 0 && J.gB >= 0)
            for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) {
                t.push_back({J.gA + 3 + i, J.gB + 3 + j, -H[i][j]});
                t.push_back({J.gB + 3 + i, J.gA + 3 + j, -H[i][j]});
            }
        return;
    }
    if (J.type == NXD_JOINT_DISTANCE_LIMIT) {
        // DistanceLimitJoint::hessian (DistanceLimitJoint.cpp:113-160)
        double C[2];
        joint_C(J, x, C);
        const bool amin = C[0] > 0.0, amax = C[1] > 0.0;
        if (!amin && !amax) return;
        const V3 pA = J.gA >= 0 ? xseg(x, J.gA) : J.pA_ref, pB = J.gB >= 0 ? xseg(x, J.gB) : J.pB_ref;
        const V3 dd = pB - pA;
        const double dist = norm(dd);
        const V3 dir = dist < 1e-12 ? mk(1, 0, 0) : dd / dist;
        double H[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int rep = 0; rep < 2; ++rep)
            if ((rep == 0 && amin) || (rep == 1 && amax))
                for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) H[i][j] += J.mu * (dir[i] * dir[j]);
        if (J.gA >= 0) for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) t.push_back({J.gA + i, J.gA + j, H[i][j]});
        if (J.gB >= 0) for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) t.push_back({J.gB + i, J.gB + j, H[i][j]});
        if (J.gA >= 0 && J.gB >= 0)
            for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) {
                t.push_back({J.gA + i, J.gB + j, -H[i][j]});
                t.push_back({J.gB + i, J.gA + j, -H[i][j]});
            }
        return;
    }
    // Joint::hessian (Joint.cpp:34-55): H = (J^T J) * mu, column-major entries
    JacRows R = joint_J(J, x);
    const size_t nc = R.cols.size();
    const int d = R.dim;
    for (size_t b = 0; b < nc; ++b)
        for (size_t a = 0; a < nc; ++a) {
            bool structural = false;
            double s = 0.0;
            for (int r = 0; r < d; ++r) {
                const double ja = R.J[r * nc + a], jb = R.J[r * nc + b];
                s += ja * jb;
                structural = true;
            }
            if (structural) t.push_back({R.cols[a], R.cols[b], s * J.mu});
        }
}
void joint_update_lambda(Joint& J, const std::vector<double>& x) {
    double C[6];
    joint_C(J, x, C);
    const int d = J.dim();
    if (J.is_limit()) {
        for (int i = 0; i < d; ++i) J.lambda[i] = std::max(0.0, J.lambda[i] + J.mu * C[i]);
    } else {
        for (int i = 0; i < d; ++i) J.lambda[i] += J.mu * C[i];
    }
}

// ---------------------------------------------------------------------------
// Velocity drive (src/Control/VelocityDriveForm.cpp:61-417), stateful as written.
// ---------------------------------------------------------------------------
double drive_effective_target(const Drive& d) {
    if (d.delay_tau <= 0.0) return d.v_target;
    if (!d.filter_init) return d.v_target;
    return d.filtered;
}
double drive_deadzone(const Drive& d, double e) {
    if (d.delay <= 0.0) return e;
    if (e > d.delay) return e - d.delay;
    if (e < -d.delay) return e + d.delay;
    return 0.0;
}
double drive_sat_torque(const Drive& d, double e) {
    const double raw = d.kv * e;
    if (!std::isfinite(d.max_torque)) return raw;
    if (d.max_torque <= 0.0) return raw;
    return d.max_torque * nxm::tanh(raw / d.max_torque);
}
// the joint coordinates a velocity drive differentiates: rotation vector
// (VelocityDriveForm) or position (LinearVelocityDriveForm::extractPosition)
V3 drive_coord(const Drive& d, const std::vector<double>& x, int g) {
    if (d.kind == NXD_DRIVE_LINEAR_VELOCITY) {
        if (g < 0 || g + 2 >= (int)x.size()) return mk(0, 0, 0);
        return xseg(x, g);
    }
    if (g < 0 || g + 5 >= (int)x.size()) return mk(0, 0, 0);
    return xseg(x, g + 3);
}
double drive_joint_velocity(Drive& d, const std::vector<double>& x) {
    const V3 tA = drive_coord(d, x, d.gA), tB = drive_coord(d, x, d.gB);
    V3 oA = mk(0, 0, 0), oB = mk(0, 0, 0);
    if (d.has_prev) {
        if (d.gA >= 0) oA = d.dt <= 0 ? mk(0, 0, 0) : (tA - d.prevA) / d.dt;
        if (d.gB >= 0) oB = d.dt <= 0 ? mk(0, 0, 0) : (tB - d.prevB) / d.dt;
    }
    const double v = dot(oB - oA, d.axis);
    d.prevA = tA; d.prevB = tB; d.has_prev = true;
    return v;
}
// 0.5 k e^2, or (m^2/k) log cosh(k e / m) with a finite limit m
// (VelocityDriveForm.cpp:300-318, LinearVelocityDriveForm.cpp:186-202,
// PositionDriveForm.cpp:117-127)
double drive_potential(const Drive& d, double e) {
    if (!std::isfinite(d.max_torque)) return 0.5 * d.kv * e * e;
    if (d.kv <= 0.0 || d.max_torque <= 0.0) return 0.0;
    const double s = (d.kv * e) / d.max_torque;
    return (d.max_torque * d.max_torque / d.kv) * nxm::log(nxm::cosh(s));
}
// PositionDriveForm::getPositionError (PositionDriveForm.cpp:66-81)
double position_error(const Drive& d, const std::vector<double>& x) {
    V3 pA = mk(0, 0, 0), pB = mk(0, 0, 0);
    if (d.gA >= 0 && d.gA + 2 < (int)x.size()) pA = xseg(x, d.gA);
    if (d.gB >= 0 && d.gB + 2 < (int)x.size()) pB = xseg(x, d.gB);
    return d.v_target - dot(pB - pA, d.axis);
}
// DampedSpringForm::springDirection (DampedSpringForm.cpp:37-46)
V3 spring_direction(const Drive& d, const std::vector<double>& x, double& length) {
    const V3 dv = xseg(x, d.gB) - xseg(x, d.gA);
    length = norm(dv);
    if (length < 1e-12) return mk(1.0, 0.0, 0.0);
    return dv / length;
}
double drive_value(nxo_world* w, Drive& d, const std::vector<double>& x) {
    (void)w;
    switch (d.kind) {
        case NXD_DRIVE_FORCE: return 0.0;
        case NXD_DRIVE_DAMPED_SPRING: {
            double len;
            (void)spring_direction(d, x, len);
            const double e = len - d.rest;
            return 0.5 * d.k * e * e;
        }
        case NXD_DRIVE_POSITION: return drive_potential(d, drive_deadzone(d, position_error(d, x)));
        default: {
            const double v = drive_joint_velocity(d, x);
            return drive_potential(d, drive_deadzone(d, drive_effective_target(d) - v));
        }
    }
}
void drive_gradient(nxo_world* w, Drive& d, const std::vector<double>& x, std::vector<double>& g) {
    switch (d.kind) {
        case NXD_DRIVE_FORCE:
            // ForceDriveForm.cpp:27-35
            if (d.gB < 0) return;
            for (int i = 0; i < 3; ++i) g[d.gB + i] -= d.force[i];
            for (int i = 0; i < 3; ++i) g[d.gB + 3 + i] -= d.torque[i];
            return;
        case NXD_DRIVE_DAMPED_SPRING: {
            // DampedSpringForm.cpp:67-82: velocities of the bodies' state
            double len;
            const V3 dir = spring_direction(d, x, len);
            const double e = len - d.rest;
            const double vrel = dot(w->bodies[d.bodyB].velocity - w->bodies[d.bodyA].velocity, dir);
            const double sc = d.k * e + d.c * vrel;
            for (int i = 0; i < 3; ++i) g[d.gB + i] += sc * dir[i];
            for (int i = 0; i < 3; ++i) g[d.gA + i] -= sc * dir[i];
            return;
        }
        case NXD_DRIVE_POSITION: {
            // PositionDriveForm.cpp:129-137
            const double f = drive_sat_torque(d, drive_deadzone(d, position_error(d, x)));
            if (d.gB >= 0) for (int i = 0; i < 3; ++i) g[d.gB + i] -= f * d.axis[i];
            if (d.gA >= 0) for (int i = 0; i < 3; ++i) g[d.gA + i] += f * d.axis[i];
            return;
        }
        case NXD_DRIVE_LINEAR_VELOCITY: {
            // LinearVelocityDriveForm.cpp:204-219
            if (d.dt <= 0.0) return;
            const double v = drive_joint_velocity(d, x);
            const double f = drive_sat_torque(d, drive_deadzone(d, drive_effective_target(d) - v));
            const double coeff = f / d.dt;
            if (d.gB >= 0) for (int i = 0; i < 3; ++i) g[d.gB + i] -= coeff * d.axis[i];
            if (d.gA >= 0) for (int i = 0; i < 3; ++i) g[d.gA + i] += coeff * d.axis[i];
            return;
        }
        default: break;
    }
    const double v = drive_joint_velocity(d, x);
    const double e = drive_deadzone(d, drive_effective_target(d) - v);
    const double tq = drive_sat_torque(d, e);
    const double dEdv = -tq;
    if (d.dt <= 0) return;
    const double dEdq = dEdv * (1.0 / d.dt);
    if (d.gB >= 0 && d.gB + 5 < (int)g.size()) for (int i = 0; i < 3; ++i) g[d.gB + 3 + i] += dEdq * d.axis[i];
    if (d.gA >= 0 && d.gA + 5 < (int)g.size()) for (int i = 0; i < 3; ++i) g[d.gA + 3 + i] -= dEdq * d.axis[i];
}
// h (a a^T) on the translation blocks: B, A, then the two off-diagonal
// blocks with -h (a a^T), entry by entry; Eigen evaluates s (a a^T) as
// (s a) a^T, so entry (i, j) is (h a_i) a_j
void push_two_body_translation(const Drive& d, double h, V3 a, std::vector<Trip>& t) {
    double H[3][3];
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) H[i][j] = (h * a[i]) * a[j];
    if (d.gB >= 0) for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) t.push_back({d.gB + i, d.gB + j, H[i][j]});
    if (d.gA >= 0) for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) t.push_back({d.gA + i, d.gA + j, H[i][j]});
    if (d.gA >= 0 && d.gB >= 0)
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                t.push_back({d.gA + i, d.gB + j, -H[i][j]});
                t.push_back({d.gB + i, d.gA + j, -H[i][j]});
            }
}
void drive_hessian(Drive& d, const std::vector<double>& x, std::vector<Trip>& t) {
    if (d.kind == NXD_DRIVE_FORCE) return;
    if (d.kind == NXD_DRIVE_DAMPED_SPRING) {
        // DampedSpringForm.cpp:84-112
        double len;
        const V3 dir = spring_direction(d, x, len);
        push_two_body_translation(d, d.k, dir, t);
        return;
    }
    if (d.kind == NXD_DRIVE_POSITION) {
        // PositionDriveForm.cpp:139-170
        double h = d.kv;
        const double err = position_error(d, x);
        if (std::isfinite(d.max_torque) && d.kv > 0.0 && d.max_torque > 0.0) {
            if (std::fabs(err) <= d.delay) h = 0.0;
            else {
                const double s = (d.kv * drive_deadzone(d, err)) / d.max_torque;
                const double th = nxm::tanh(s);
                h = d.kv * (1.0 - th * th);
            }
        }
        if (h == 0.0) return;
        push_two_body_translation(d, h, d.axis, t);
        return;
    }
    if (d.dt <= 0) return;
    double H = d.kv / (d.dt * d.dt);
    if (std::isfinite(d.max_torque) && d.kv > 0.0 && d.max_torque > 0.0) {
        const double v = drive_joint_velocity(d, x);
        const double e = drive_effective_target(d) - v;
        if (std::fabs(e) <= d.delay) H = 0.0;
        else {
            const double ee = drive_deadzone(d, e);
            const double s = (d.kv * ee) / d.max_torque;
            const double th = nxm::tanh(s);
            H = (d.kv * (1.0 - th * th)) / (d.dt * d.dt);
        }
    }
    if (H == 0.0) return;
    if (d.kind == NXD_DRIVE_LINEAR_VELOCITY) {
        // LinearVelocityDriveForm.cpp:221-270
        push_two_body_translation(d, H, d.axis, t);
        return;
    }
    for (int side = 0; side < 2; ++side) {
        const int g = side == 0 ? d.gB : d.gA;
        if (g < 0) continue;
        const int r = g + 3;
        for (int i = 0; i < 3; ++i) t.push_back({r + i, r + i, H * d.axis[i] * d.axis[i]});
        for (int i = 0; i < 3; ++i)
            for (int j = i + 1; j < 3; ++j) {
                const double od = H * d.axis[i] * d.axis[j];
                t.push_back({r + i, r + j, od});
                t.push_back({r + j, r + i, od});
            }
    }
}

// ---------------------------------------------------------------------------
// Contact forms
// ---------------------------------------------------------------------------
// DistanceBarrierForm::contactDistance (DistanceBarrierForm.cpp:88-99)
inline double contact_distance(const Contact& c, const std::vector<double>& x) {
    const V3 pA = xseg(x, c.bodyA * 6), pB = xseg(x, c.bodyB * 6);
    return std::max(1e-9, dot(pB - pA, c.normal));
}
double barrier_form_value(nxo_world* w, const std::vector<double>& x) {
    std::vector<double> ev;
    for (const auto& c : w->barrier_contacts) ev.push_back(barrier_value(contact_distance(c, x), w->barrier_dhat, w->barrier_kappa));
    return tree_sum(ev);
}
void barrier_form_gradient(nxo_world* w, const std::vector<double>& x, std::vector<double>& g) {
    std::fill(g.begin(), g.end(), 0.0);
    for (const auto& c : w->barrier_contacts) {
        const double d = contact_distance(c, x);
        if (d >= w->barrier_dhat) continue;
        const int a = c.bodyA * 6, b = c.bodyB * 6;
        const double gp = barrier_gradient(d, w->barrier_dhat, w->barrier_kappa);
        const V3 ga = -gp * c.normal, gb = gp * c.normal;
        for (int i = 0; i < 3; ++i) { g[a + i] += ga[i]; g[b + i] += gb[i]; }
    }
}
void barrier_form_hessian(nxo_world* w, const std::vector<double>& x, std::vector<Trip>& t) {
    for (const auto& c : w->barrier_contacts) {
        const double d = contact_distance(c, x);
        if (d >= w->barrier_dhat) continue;
        const int a = c.bodyA * 6, b = c.bodyB * 6;
        const double h = barrier_hessian(d, w->barrier_dhat, w->barrier_kappa);
        for (int r = 0; r < 3; ++r)
            for (int cc = 0; cc < 3; ++cc) {
                const double blk = h * (c.normal[r] * c.normal[cc]);
                t.push_back({a + r, a + cc, blk});
                t.push_back({b + r, b + cc, blk});
                t.push_back({a + r, b + cc, -blk});
                t.push_back({b + r, a + cc, -blk});
            }
    }
}
std::vector<double> barrier_normal_forces(nxo_world* w, const std::vector<double>& x) {
    std::vector<double> nf;
    nf.reserve(w->barrier_contacts.size());
    for (const auto& c : w->barrier_contacts) {
        const double d = contact_distance(c, x);
        if (d < w->barrier_dhat && d > 0.0) nf.push_back(std::fabs(barrier_gradient(d, w->barrier_dhat, w->barrier_kappa)));
        else nf.push_back(0.0);
    }
    return nf;
}

// FrictionPotential (src/Physics/Contact/Friction.cpp:5-61)
double fric_value(V3 u, double N, double mu, double eps) {
    if (N <= 0) return 0.0;
    const double un = norm(u);
    const double sn = std::sqrt(un * un + eps * eps);
    return mu * N * (sn - eps);
}
V3 fric_gradient(V3 u, double N, double mu, double eps) {
    if (N <= 0) return mk(0, 0, 0);
    const double un = norm(u);
    if (un < 1e-12) return mk(0, 0, 0);
    const double sn = std::sqrt(un * un + eps * eps);
    const double sc = mu * N / sn;
    return sc * u;
}
M3 fric_hessian(V3 u, double N, double mu, double eps) {
    M3 H;
    if (N <= 0) { for (double& v : H.m) v = 0; return H; }
    const double un = norm(u);
    if (un < 1e-12) {
        const double s = mu * N / eps;
        for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) H(i, j) = (i == j) ? s : 0.0;
        return H;
    }
    const double sn = std::sqrt(un * un + eps * eps);
    const double sc = mu * N / sn;
    const double s2 = sn * sn;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) H(i, j) = sc * ((i == j ? 1.0 : 0.0) - u[i] * u[j] / s2);
    return H;
}

// FrictionForm helpers (src/Dynamics/Forms/FrictionForm.cpp:174-224)
struct FricGeom { V3 rA, rB; M3 P; V3 n; };
FricGeom fric_geom(nxo_world* w, const Contact& c, const std::vector<double>& x) {
    FricGeom G;
    const Body& A = w->bodies[c.bodyA];
    const Body& B = w->bodies[c.bodyB];
    const Q rotA = update_rotation_gt(A.orientation, xseg(x, c.bodyA * 6 + 3));
    const Q rotB = update_rotation_gt(B.orientation, xseg(x, c.bodyB * 6 + 3));
    const V3 lA = qrot(qconj(A.orientation), c.point - A.position);
    const V3 lB = qrot(qconj(B.orientation), c.point - B.position);
    G.rA = qrot(rotA, lA);
    G.rB = qrot(rotB, lB);
    G.n = sqnorm(c.normal) > 1e-16 ? normalized(c.normal) : mk(0, 1, 0);
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) G.P(i, j) = (i == j ? 1.0 : 0.0) - G.n[i] * G.n[j];
    return G;
}
V3 fric_tangent_disp(nxo_world* w, const Contact& c, const std::vector<double>& x) {
    const FricGeom G = fric_geom(w, c, x);
    const Body& A = w->bodies[c.bodyA];
    const Body& B = w->bodies[c.bodyB];
    const V3 dA = xseg(x, c.bodyA * 6) - A.position, dB = xseg(x, c.bodyB * 6) - B.position;
    V3 oA = mk(0, 0, 0), oB = mk(0, 0, 0), vA = mk(0, 0, 0), vB = mk(0, 0, 0);
    const double dt = w->friction_dt;
    if (dt > 1e-12) {
        oA = xseg(x, c.bodyA * 6 + 3) / dt; oB = xseg(x, c.bodyB * 6 + 3) / dt;
        vA = dA / dt; vB = dB / dt;
    }
    vA = vA + cross(oA, G.rA);
    vB = vB + cross(oB, G.rB);
    const V3 rel = vB - vA;
    const V3 tv = rel - dot(rel, G.n) * G.n;
    return tv * dt;
}
// J_A = [-P, P [rA]x], J_B = [P, -P [rB]x] as 3x6
void fric_jacobians(const FricGeom& G, double JA[3][6], double JB[3][6]) {
    const M3 sA = cross_mat(G.rA), sB = cross_mat(G.rB);
    const M3 PA = mat_mul(G.P, sA), PB = mat_mul(G.P, sB);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            JA[i][j] = -G.P(i, j); JB[i][j] = G.P(i, j);
            JA[i][3 + j] = PA(i, j); JB[i][3 + j] = -PB(i, j);
        }
}
double friction_form_value(nxo_world* w, const std::vector<double>& x) {
    std::vector<double> ev(w->friction_contacts.size(), 0.0);
    for (size_t i = 0; i < w->friction_contacts.size(); ++i) {
        if (i >= w->normal_forces.size()) continue;
        const double N = w->normal_forces[i];
        if (N <= 0) continue;
        ev[i] = fric_value(fric_tangent_disp(w, w->friction_contacts[i], x), N, w->friction_mu, w->friction_eps);
    }
    return tree_sum(ev);
}
void friction_form_gradient(nxo_world* w, const std::vector<double>& x, std::vector<double>& g) {
    std::fill(g.begin(), g.end(), 0.0);
    for (size_t i = 0; i < w->friction_contacts.size(); ++i) {
        if (i >= w->normal_forces.size()) continue;
        const double N = w->normal_forces[i];
        if (N <= 0) continue;
        const Contact& c = w->friction_contacts[i];
        const V3 fg = fric_gradient(fric_tangent_disp(w, c, x), N, w->friction_mu, w->friction_eps);
        const FricGeom G = fric_geom(w, c, x);
        double JA[3][6], JB[3][6];
        fric_jacobians(G, JA, JB);
        for (int k = 0; k < 6; ++k) {
            g[c.bodyA * 6 + k] += JA[0][k] * fg.x + JA[1][k] * fg.y + JA[2][k] * fg.z;
            g[c.bodyB * 6 + k] += JB[0][k] * fg.x + JB[1][k] * fg.y + JB[2][k] * fg.z;
        }
    }
}
void friction_form_hessian(nxo_world* w, const std::vector<double>& x, std::vector<Trip>& t) {
    for (size_t i = 0; i < w->friction_contacts.size(); ++i) {
        if (i >= w->normal_forces.size()) continue;
        const double N = w->normal_forces[i];
        if (N <= 0) continue;
        const Contact& c = w->friction_contacts[i];
        const M3 Hf = fric_hessian(fric_tangent_disp(w, c, x), N, w->friction_mu, w->friction_eps);
        const FricGeom G = fric_geom(w, c, x);
        double JA[3][6], JB[3][6];
        fric_jacobians(G, JA, JB);
        // H_XY = J_X^T Hf J_Y evaluated as (J_X^T Hf) J_Y
        auto block = [&](double Jx[3][6], double Jy[3][6], double out[6][6]) {
            double T[6][3];
            for (int r = 0; r < 6; ++r)
                for (int k = 0; k < 3; ++k) T[r][k] = Jx[0][r] * Hf(0, k) + Jx[1][r] * Hf(1, k) + Jx[2][r] * Hf(2, k);
            for (int r = 0; r < 6; ++r)
                for (int cc = 0; cc < 6; ++cc) out[r][cc] = T[r][0] * Jy[0][cc] + T[r][1] * Jy[1][cc] + T[r][2] * Jy[2][cc];
        };
        double AA[6][6], BB[6][6], AB[6][6], BA[6][6];
        block(JA, JA, AA); block(JB, JB, BB); block(JA, JB, AB); block(JB, JA, BA);
        const int a = c.bodyA * 6, b = c.bodyB * 6;
        for (int r = 0; r < 6; ++r)
            for (int cc = 0; cc < 6; ++cc) {
                t.push_back({a + r, a + cc, AA[r][cc]});
                t.push_back({b + r, b + cc, BB[r][cc]});
                t.push_back({a + r, b + cc, AB[r][cc]});
                t.push_back({b + r, a + cc, BA[r][cc]});
            }
    }
}

// ---------------------------------------------------------------------------
// SimulationProblem (IPCSolver.cpp:137-262)
// ---------------------------------------------------------------------------
double inertia_value(nxo_world* w, const std::vector<double>& x) {
    std::vector<double> ev(w->bodies.size());
    for (size_t i = 0; i < w->bodies.size(); ++i) {
        const int idx = (int)i * 6;
        const V3 dp = xseg(x, idx) - xseg(w->x_hat, idx);
        const double et = 0.5 * w->bodies[i].mass * sqnorm(dp);
        const V3 dth = xseg(x, idx + 3) - xseg(w->x_hat, idx + 3);
        const M3& I = w->bodies[i].inertia;
        // (d^T I) d
        const V3 r = mk(dth.x * I(0, 0) + dth.y * I(1, 0) + dth.z * I(2, 0),
                        dth.x * I(0, 1) + dth.y * I(1, 1) + dth.z * I(2, 1),
                        dth.x * I(0, 2) + dth.y * I(1, 2) + dth.z * I(2, 2));
        ev[i] = et + 0.5 * dot(r, dth);
    }
    return tree_sum(ev);
}
void inertia_gradient(nxo_world* w, const std::vector<double>& x, std::vector<double>& g) {
    for (size_t i = 0; i < w->bodies.size(); ++i) {
        const int idx = (int)i * 6;
        const V3 gp = w->bodies[i].mass * (xseg(x, idx) - xseg(w->x_hat, idx));
        const V3 gr = mul(w->bodies[i].inertia, xseg(x, idx + 3) - xseg(w->x_hat, idx + 3));
        for (int k = 0; k < 3; ++k) { g[idx + k] = gp[k]; g[idx + 3 + k] = gr[k]; }
    }
}
void inertia_hessian(nxo_world* w, std::vector<Trip>& t) {
    for (size_t i = 0; i < w->bodies.size(); ++i) {
        const int idx = (int)i * 6;
        const double m = w->bodies[i].mass;
        t.push_back({idx, idx, m}); t.push_back({idx + 1, idx + 1, m}); t.push_back({idx + 2, idx + 2, m});
        for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) t.push_back({idx + 3 + a, idx + 3 + b, w->bodies[i].inertia(a, b)});
    }
}
const V3 kGravity = mk(0, -9.81, 0);
double gravity_value(nxo_world* w, const std::vector<double>& x) {
    std::vector<double> ev(w->bodies.size());
    for (size_t i = 0; i < w->bodies.size(); ++i) ev[i] = -(w->bodies[i].mass * dot(kGravity, xseg(x, (int)i * 6)));
    return tree_sum(ev);
}
void gravity_gradient(nxo_world* w, std::vector<double>& g) {
    for (size_t i = 0; i < w->bodies.size(); ++i) {
        const V3 f = -w->bodies[i].mass * kGravity;
        for (int k = 0; k < 3; ++k) { g[i * 6 + k] = f[k]; g[i * 6 + 3 + k] = 0.0; }
    }
}
double constraint_value(nxo_world* w, const std::vector<double>& x) {
    std::vector<double> ev;
    for (const auto& J : w->joints) ev.push_back(joint_value(J, x));
    return tree_sum(ev);
}
double drives_value(nxo_world* w, const std::vector<double>& x) {
    std::vector<double> ev;
    for (auto& d : w->drives) ev.push_back(drive_value(w, d, x));
    return tree_sum(ev);
}

// acceleration_scaling: ImplicitEuler dt^2 (ImplicitEulerIntegrator.cpp:9-11),
// ImplicitNewmark beta dt^2 (ImplicitNewmark.cpp:12-14)
double scaling(nxo_world* w) {
    if (w->s.integrator == NXD_INTEGRATOR_IMPLICIT_NEWMARK) return (w->s.newmark_beta * w->dt) * w->dt;
    return w->dt * w->dt;
}

double problem_value(nxo_world* w, const std::vector<double>& x) {
    double v = inertia_value(w, x);
    const double s = scaling(w);
    v += s * gravity_value(w, x);
    v += constraint_value(w, x);
    // world.forms: drives, then barrier (if pushed), then friction
    for (auto& d : w->drives) v += s * drive_value(w, d, x);
    if (w->barrier_in_forms) v += s * barrier_form_value(w, x);
    if (w->friction_form) v += s * friction_form_value(w, x);
    return v;
}
void problem_gradient(nxo_world* w, const std::vector<double>& x, std::vector<double>& g) {
    const size_t n = x.size();
    g.assign(n, 0.0);
    std::vector<double> t(n, 0.0);
    const double s = scaling(w);
    inertia_gradient(w, x, t);
    for (size_t i = 0; i < n; ++i) g[i] += t[i];
    std::fill(t.begin(), t.end(), 0.0);
    gravity_gradient(w, t);
    for (size_t i = 0; i < n; ++i) g[i] += s * t[i];
    std::fill(t.begin(), t.end(), 0.0);
    for (const auto& J : w->joints) joint_gradient(J, x, t);
    for (size_t i = 0; i < n; ++i) g[i] += t[i];
    for (auto& d : w->drives) {
        std::fill(t.begin(), t.end(), 0.0);
        drive_gradient(w, d, x, t);
        for (size_t i = 0; i < n; ++i) g[i] += s * t[i];
    }
    if (w->barrier_in_forms) {
        barrier_form_gradient(w, x, t);
        for (size_t i = 0; i < n; ++i) g[i] += s * t[i];
    }
    if (w->friction_form) {
        friction_form_gradient(w, x, t);
        for (size_t i = 0; i < n; ++i) g[i] += s * t[i];
    }
}
void problem_hessian(nxo_world* w, const std::vector<double>& x, std::vector<Trip>& trips) {
    trips.clear();
    const double s = scaling(w);
    inertia_hessian(w, trips);
    std::vector<Trip> tmp;
    for (const auto& J : w->joints) joint_hessian(J, x, tmp);
    for (const auto& t : tmp) trips.push_back(t);
    for (auto& d : w->drives) {
        tmp.clear();
        drive_hessian(d, x, tmp);
        for (const auto& t : tmp) trips.push_back({t.r, t.c, t.v * s});
    }
    if (w->barrier_in_forms) {
        tmp.clear();
        barrier_form_hessian(w, x, tmp);
        for (const auto& t : tmp) trips.push_back({t.r, t.c, t.v * s});
    }
    if (w->friction_form) {
        tmp.clear();
        friction_form_hessian(w, x, tmp);
        for (const auto& t : tmp) trips.push_back({t.r, t.c, t.v * s});
    }
}
double problem_contact_value(nxo_world* w, const std::vector<double>& x) {
    double v = 0.0;
    const double s = scaling(w);
    if (w->barrier_in_forms) v += s * barrier_form_value(w, x);
    if (w->friction_form) v += s * friction_form_value(w, x);
    return v;
}
void problem_contact_gradient(nxo_world* w, const std::vector<double>& x, std::vector<double>& g) {
    const size_t n = x.size();
    g.assign(n, 0.0);
    std::vector<double> t(n, 0.0);
    const double s = scaling(w);
    if (w->barrier_in_forms) {
        barrier_form_gradient(w, x, t);
        for (size_t i = 0; i < n; ++i) g[i] += s * t[i];
    }
    if (w->friction_form) {
        friction_form_gradient(w, x, t);
        for (size_t i = 0; i < n; ++i) g[i] += s * t[i];
    }
}

// ---------------------------------------------------------------------------
// Linear solve: triplets -> 6x6 blocks (duplicates summed in triplet order,
// as setFromTriplets) -> connected components -> dense LDL^T each, using
// the lower triangle (Eigen SimplicialLDLT default UpLo = Lower).
// ---------------------------------------------------------------------------
struct BlockMatrix {
    int nb = 0;
    std::unordered_map<long long, std::array<double, 36>> blocks;
    std::array<double, 36>& at(int r, int c) {
        long long key = (long long)r * nb + c;
        auto it = blocks.find(key);
        if (it == blocks.end()) { std::array<double, 36> z{}; it = blocks.emplace(key, z).first; }
        return it->second;
    }
};
int find_root(std::vector<int>& p, int a) { while (p[a] != a) { p[a] = p[p[a]]; a = p[a]; } return a; }

// returns false on an exactly zero pivot
bool ldlt_dense(std::vector<double>& A, int n) {
    // in place: L strictly lower, D on the diagonal; reads A(i,j) for i >= j only
    std::vector<double> d(n);
    for (int j = 0; j < n; ++j) {
        double dj = A[(size_t)j * n + j];
        for (int k = 0; k < j; ++k) { const double l = A[(size_t)j * n + k]; dj -= l * l * d[k]; }
        if (dj == 0.0) return false;
        d[j] = dj;
        A[(size_t)j * n + j] = dj;
        for (int i = j + 1; i < n; ++i) {
            double s = A[(size_t)i * n + j];
            for (int k = 0; k < j; ++k) s -= A[(size_t)i * n + k] * A[(size_t)j * n + k] * d[k];
            A[(size_t)i * n + j] = s / dj;
        }
    }
    return true;
}
void ldlt_solve_dense(const std::vector<double>& A, int n, std::vector<double>& b) {
    for (int i = 0; i < n; ++i) {
        double s = b[i];
        for (int k = 0; k < i; ++k) s -= A[(size_t)i * n + k] * b[k];
        b[i] = s;
    }
    for (int i = 0; i < n; ++i) b[i] /= A[(size_t)i * n + i];
    // backward substitution; each x_i takes its updates in descending k
    // (the column-oriented order)
    for (int i = n - 1; i >= 0; --i) {
        double s = b[i];
        for (int k = n - 1; k > i; --k) s -= A[(size_t)k * n + i] * b[k];
        b[i] = s;
    }
}

bool solve_system(int ndof, const std::vector<Trip>& trips, const std::vector<double>& rhs, std::vector<double>& sol) {
    const int nb = ndof / 6;
    BlockMatrix H;
    H.nb = nb;
    for (const auto& t : trips) H.at(t.r / 6, t.c / 6)[(t.r % 6) * 6 + (t.c % 6)] += t.v;
    std::vector<int> parent(nb);
    std::iota(parent.begin(), parent.end(), 0);
    for (const auto& kv : H.blocks) {
        const int r = (int)(kv.first / nb), c = (int)(kv.first % nb);
        if (r != c) { int a = find_root(parent, r), b = find_root(parent, c); if (a != b) parent[std::max(a, b)] = std::min(a, b); }
    }
    std::unordered_map<int, std::vector<int>> comps;
    for (int i = 0; i < nb; ++i) comps[find_root(parent, i)].push_back(i);
    sol.assign(ndof, 0.0);
    for (auto& kv : comps) {
        // members ordered by (number of distinct coupled bodies, index): leaves
        // of stars and the ends of chains come first, so they factor without
        // fill; the device solver uses the same order
        std::vector<int> members = kv.second;   // ascending
        if (members.size() > 1) {
            std::vector<std::pair<int, int>> key;
            for (int b : members) {
                int deg = 0;
                for (int o : members)
                    if (o != b && (H.blocks.count((long long)b * nb + o) || H.blocks.count((long long)o * nb + b))) ++deg;
                key.push_back({deg, b});
            }
            std::sort(key.begin(), key.end());
            for (size_t t = 0; t < key.size(); ++t) members[t] = key[t].second;
        }
        const int m = (int)members.size(), n = 6 * m;
        std::vector<double> A((size_t)n * n, 0.0);
        for (int bi = 0; bi < m; ++bi)
            for (int bj = 0; bj <= bi; ++bj) {
                auto it = H.blocks.find((long long)members[bi] * nb + members[bj]);
                if (it == H.blocks.end()) continue;
                for (int r = 0; r < 6; ++r)
                    for (int c = 0; c < 6; ++c) {
                        const int gi = bi * 6 + r, gj = bj * 6 + c;
                        if (gi >= gj) A[(size_t)gi * n + gj] = it->second[r * 6 + c];
                    }
            }
        if (!ldlt_dense(A, n)) return false;
        std::vector<double> b(n);
        for (int bi = 0; bi < m; ++bi) for (int r = 0; r < 6; ++r) b[bi * 6 + r] = rhs[members[bi] * 6 + r];
        ldlt_solve_dense(A, n, b);
        for (int bi = 0; bi < m; ++bi) for (int r = 0; r < 6; ++r) sol[members[bi] * 6 + r] = b[bi * 6 + r];
    }
    return true;
}

// ---------------------------------------------------------------------------
// NewtonSolver::minimize (src/Math/NewtonSolver.cpp:10-95) with
// BacktrackingLineSearch::search (src/Math/LineSearch.cpp:6-58)
// ---------------------------------------------------------------------------
double line_search(nxo_world* w, const std::vector<double>& x, const std::vector<double>& dir, const std::vector<double>& grad,
                   const std::vector<double>& cgrad, double alpha0) {
    const nxd_settings& s = w->s;
    double alpha = alpha0;
    const double fx = problem_value(w, x);
    std::vector<double> prod(x.size());
    for (size_t i = 0; i < x.size(); ++i) prod[i] = grad[i] * dir[i];
    const double descent = tree_sum(prod);
    const double fc = problem_contact_value(w, x);
    for (size_t i = 0; i < x.size(); ++i) prod[i] = cgrad[i] * dir[i];
    const double cdesc = tree_sum(prod);
    if (descent > 0) return 0.0;
    std::vector<double> xn(x.size());
    for (int it = 0; it < s.ls_max_iters; ++it) {
        for (size_t i = 0; i < x.size(); ++i) xn[i] = x[i] + alpha * dir[i];
        const double fn = problem_value(w, xn);
        const double fcn = problem_contact_value(w, xn);
        bool cok = cdesc <= 0.0 ? (fcn <= fc + s.ls_c1 * alpha * cdesc) : (fcn <= fc);
        if (fn <= fx + s.ls_c1 * alpha * descent && cok) return alpha;
        alpha *= s.ls_rho;
    }
    return 0.0;
}

bool newton_minimize(nxo_world* w, std::vector<double>& x, int* iters_out) {
    const nxd_settings& s = w->s;
    std::vector<double> grad, cgrad, dx;
    std::vector<Trip> trips;
    const size_t n = x.size();
    for (int iter = 0; iter < s.newton_max_iters; ++iter) {
        *iters_out = iter;
        problem_gradient(w, x, grad);
        double ginf = 0.0;
        for (double v : grad) ginf = std::max(ginf, std::fabs(v));
        if (ginf < s.newton_tol) return true;
        problem_hessian(w, x, trips);
        std::vector<double> rhs(n);
        for (size_t i = 0; i < n; ++i) rhs[i] = -grad[i];
        if (!solve_system((int)n, trips, rhs, dx)) return false;
        const double init_alpha = std::min(1.0, 1.0);   // OptimizationProblem::maxStep == 1
        problem_contact_gradient(w, x, cgrad);
        (void)problem_contact_value(w, x);              // contact_value_before (diagnostic)
        const double alpha = line_search(w, x, dx, grad, cgrad, init_alpha);
        if (alpha == 0.0) { w->diag.line_search_failures++; return false; }
        for (size_t i = 0; i < n; ++i) x[i] = x[i] + alpha * dx[i];
        (void)problem_contact_value(w, x);              // contact_value_after (diagnostic)
    }
    *iters_out = s.newton_max_iters;
    return false;
}

// ---------------------------------------------------------------------------
// IPCSolver::step (IPCSolver.cpp:808-1231)
// ---------------------------------------------------------------------------
void initialize_adaptive_barrier(nxo_world* w) {
    // IPCSolver::initializeAdaptiveBarrier (IPCSolver.cpp:327-353) + AdaptiveBarrier::initialize
    if (w->bodies.empty()) return;
    std::vector<double> masses;
    V3 bmin = mk(kInf, kInf, kInf), bmax = mk(-kInf, -kInf, -kInf);
    for (const auto& b : w->bodies) { masses.push_back(b.mass); bmin = cwmin(bmin, b.position); bmax = cwmax(bmax, b.position); }
    const double tm = tree_sum(masses);
    const double am = tm / (double)w->bodies.size();
    double diag = norm(bmax - bmin);
    if (diag < 1e-6) diag = 1.0;
    w->kappa_min = 1e11 * am / (diag * diag);
    w->kappa = w->kappa_min;
    w->dhat = 1e-3;   // AdaptiveBarrierParams::initial_dhat
}

int body_index_of_id(nxo_world* w, int id) {
    for (int i = 0; i < (int)w->bodies.size(); ++i) if (w->bodies[i].id == id) return i;
    return -1;
}

void step(nxo_world* w, double dt) {
    const double t0 = now_s();
    const nxd_settings& s = w->s;
    w->diag.line_search_failures = 0;
    assembler_build(w);
    build_candidate_set(w, w->dhat, w->cand);
    const double t1 = now_s();

    if (s.enable_adaptive_barrier) {
        if (!w->barrier_initialized) { initialize_adaptive_barrier(w); w->barrier_initialized = true; }
        const double dh = w->dhat;
        double bmd = estimate_min_body_pair_distance(w, dh * 2.0);
        if (!std::isfinite(bmd)) bmd = kInf;
        if (bmd < dh * 2.0) {
            const double md = w->literal_min_distance ? scene_min_distance_literal(w) : scene_min_distance_pruned(w);
            w->diag.scene_min_distance = md;
            if (md < kInf) {
                // AdaptiveBarrier::updateStiffness (AdaptiveBarrier.h:33-37)
                if (md < 1e-9 && w->kappa < 1e20) w->kappa = std::min(w->kappa * 2.0, 1e20);
            }
        }
    }
    const double t2 = now_s();

    double actual_dt = dt;
    if (s.enable_ccd) actual_dt = compute_max_step(w, dt);
    w->diag.actual_dt = actual_dt;
    const double t3 = now_s();

    const int N = (int)w->bodies.size();
    const int n = N * 6;
    std::vector<double> x(n, 0.0), v(n, 0.0), a(n, 0.0);
    for (int i = 0; i < N; ++i) {
        const Body& b = w->bodies[i];
        for (int k = 0; k < 3; ++k) {
            x[i * 6 + k] = b.position[k]; x[i * 6 + 3 + k] = 0.0;
            v[i * 6 + k] = b.velocity[k]; v[i * 6 + 3 + k] = b.angular_velocity[k];
            a[i * 6 + k] = b.linear_acceleration[k]; a[i * 6 + 3 + k] = b.angular_acceleration[k];
        }
    }
    // ImplicitTimeIntegrator::init + x_tilde (ImplicitEulerIntegrator.cpp:5-7,
    // ImplicitNewmark.cpp:8-10)
    w->x_prev = x; w->v_prev = v; w->a_prev = a; w->dt = actual_dt;
    const bool newmark = s.integrator == NXD_INTEGRATOR_IMPLICIT_NEWMARK;
    const double nm_s1 = (actual_dt * actual_dt) * (0.5 - s.newmark_beta);
    std::vector<double> x_hat(n);
    for (int i = 0; i < n; ++i) {
        x_hat[i] = x[i] + actual_dt * v[i];
        if (newmark) x_hat[i] = x_hat[i] + nm_s1 * a[i];
    }
    std::vector<double> x_new = x_hat;
    w->x_hat = x_hat;

    std::vector<Contact> active;
    const bool needs = s.enable_adaptive_barrier || (s.enable_friction && s.friction_coeff > 0.0);
    int raw = 0;
    if (needs) active = detect_contacts(w, nullptr, &raw);
    w->diag.n_contacts_raw = raw;
    w->diag.n_contacts = (int)active.size();
    w->barrier_form = needs;
    w->barrier_in_forms = false;
    w->friction_form = false;
    if (needs) {
        w->barrier_dhat = std::max(1e-9, w->dhat);
        w->barrier_kappa = std::max(0.0, w->kappa);
        w->barrier_contacts = active;
    } else {
        w->barrier_contacts.clear();
    }
    if (s.enable_adaptive_barrier && w->barrier_form) w->barrier_in_forms = true;
    if (s.enable_friction && s.friction_coeff > 0) {
        w->friction_form = true;
        // effective coefficient with per-pair overrides (IPCSolver.cpp:891-911)
        double mu = s.friction_coeff;
        if (!active.empty() && !w->pair_friction.empty()) {
            double sum = 0.0;
            int cnt = 0;
            for (const Contact& c : active) {
                auto it = w->pair_friction.find(nxo_world::pair_key(w->bodies[c.bodyA].id, w->bodies[c.bodyB].id));
                sum += it != w->pair_friction.end() ? it->second : s.friction_coeff;
                ++cnt;
            }
            if (cnt > 0) mu = sum / (double)cnt;
        }
        w->friction_mu = mu;
        w->friction_eps = 1e-8;
        w->friction_dt = std::max(0.0, actual_dt);
        w->friction_contacts = active;
        w->normal_forces.clear();
    }
    if (w->barrier_form) { w->barrier_dhat = std::max(1e-9, w->dhat); w->barrier_kappa = std::max(0.0, w->kappa); }
    // drives: setTimeStep, advanceControlState, updateGlobalIndices (IPCSolver.cpp:923-958)
    for (auto& d : w->drives) {
        d.dt = actual_dt;
        if (d.delay_tau <= 0.0) { d.filtered = d.v_target; d.filter_init = false; }
        else if (!d.filter_init) { d.filtered = d.v_target; d.filter_init = true; }
        else if (d.dt > 0.0) { const double al = d.dt / (d.delay_tau + d.dt); d.filtered += al * (d.v_target - d.filtered); }
        d.gA = d.bodyA >= 0 ? d.bodyA * 6 : -1;
        d.gB = d.bodyB >= 0 ? d.bodyB * 6 : -1;
        d.has_prev = false;
    }
    const double t4 = now_s();

    w->diag.last_max_constraint_violation = 0.0;
    w->diag.last_dual_residual = 0.0;
    w->diag.last_contact_residual = 0.0;
    int newton_total = 0;
    int alm_run = 0;
    bool conv_last = false;
    for (int alm = 0; alm < s.alm_max_iters; ++alm) {
        alm_run = alm + 1;
        for (auto& J : w->joints) {
            // updateState dispatch (IPCSolver.cpp:966-1066): step-start poses
            const int ia = body_index_of_id(w, J.bodyA_id);
            if (J.type == NXD_JOINT_FIXED) {
                J.gA = ia * 6; J.qA_ref = w->bodies[ia].orientation;
            } else {
                const int ib = body_index_of_id(w, J.bodyB_id);
                J.gA = ia * 6; J.gB = ib * 6;
                J.pA_ref = w->bodies[ia].position; J.qA_ref = w->bodies[ia].orientation;
                J.pB_ref = w->bodies[ib].position; J.qB_ref = w->bodies[ib].orientation;
            }
        }
        int it = 0;
        const bool converged = newton_minimize(w, x_new, &it);
        newton_total += it;
        conv_last = converged;

        double mcv = 0.0, dual = 0.0;
        for (auto& J : w->joints) {
            double C[6];
            joint_C(J, x_new, C);
            const int d = J.dim();
            if (d > 0) {
                double inf = 0.0;
                for (int k = 0; k < d; ++k) inf = std::max(inf, std::fabs(C[k]));
                mcv = std::max(mcv, inf);
                const double dc = J.mu * inf;
                if (std::isfinite(dc)) dual = std::max(dual, std::min(dc, 1e12));
                else dual = std::max(dual, 1e12);
                if (inf > s.alm_hardening_trigger * s.alm_constraint_tol) {
                    const double ns = J.mu * s.alm_hardening_ratio;
                    J.mu = std::isfinite(ns) ? std::min(ns, 1e12) : 1e12;
                }
            }
        }
        for (auto& J : w->joints) joint_update_lambda(J, x_new);

        if (w->barrier_form || w->friction_form) {
            int rc = 0;
            const auto ic = detect_contacts(w, &x_new, &rc);
            w->diag.n_contacts_raw = rc;
            w->diag.n_contacts = (int)ic.size();
            if (w->barrier_form) w->barrier_contacts = ic;
            if (s.enable_friction && w->friction_form) {
                w->friction_contacts = ic;
                if (w->barrier_form) w->normal_forces = barrier_normal_forces(w, x_new);
                else w->normal_forces.assign(ic.size(), 0.0);
            }
        }
        double cres = 0.0;
        if (w->barrier_form || w->friction_form) {
            std::vector<double> cg(n, 0.0), t(n, 0.0);
            if (w->barrier_form) { barrier_form_gradient(w, x_new, t); for (int i = 0; i < n; ++i) cg[i] += t[i]; }
            if (s.enable_friction && w->friction_form) { friction_form_gradient(w, x_new, t); for (int i = 0; i < n; ++i) cg[i] += t[i]; }
            if (n > 0) {
                for (double vv : cg) cres = std::max(cres, std::fabs(vv));
                if (!std::isfinite(cres)) cres = 1e12;
            }
        }
        w->diag.last_max_constraint_violation = mcv;
        w->diag.last_dual_residual = dual;
        w->diag.last_contact_residual = cres;
        if (converged && mcv <= s.alm_constraint_tol && dual <= s.alm_dual_tol && cres <= s.alm_contact_tol) break;
    }
    w->diag.alm_iterations = alm_run;
    w->diag.newton_iterations = newton_total;
    w->diag.newton_converged = conv_last ? 1 : 0;
    const double t5 = now_s();

    // update_quantities (ImplicitEulerIntegrator.cpp:13-25, ImplicitNewmark.cpp:16-30)
    // + write-back (IPCSolver.cpp:1168-1195)
    std::vector<double> vn(n), an(n);
    if (newmark) {
        const double den = (s.newmark_beta * actual_dt) * actual_dt;
        for (int i = 0; i < n; ++i) an[i] = (x_new[i] - w->x_hat[i]) / den;
        for (int i = 0; i < n; ++i)
            vn[i] = w->v_prev[i] + actual_dt * ((1.0 - s.newmark_gamma) * w->a_prev[i] + s.newmark_gamma * an[i]);
    } else {
        for (int i = 0; i < n; ++i) vn[i] = (x_new[i] - w->x_prev[i]) / actual_dt;
        for (int i = 0; i < n; ++i) an[i] = (vn[i] - w->v_prev[i]) / actual_dt;
    }
    for (int i = 0; i < N; ++i) {
        Body& b = w->bodies[i];
        const int idx = i * 6;
        b.linear_acceleration = xseg(an, idx);
        b.angular_acceleration = xseg(an, idx + 3);
        b.velocity = xseg(vn, idx);
        b.angular_velocity = xseg(vn, idx + 3);
        b.position = xseg(x_new, idx);
        b.orientation = update_rotation_gt(b.orientation, xseg(x_new, idx + 3));
    }
    // drive KPIs (IPCSolver.cpp:1197-1215)
    double max_vw = 0.0;
    int dc = 0, sat = 0;
    for (auto& d : w->drives) {
        if (d.kind != NXD_DRIVE_ANGULAR_VELOCITY) continue;   // VelocityDriveForms only
        ++dc;
        V3 oA = d.bodyA >= 0 ? w->bodies[d.bodyA].angular_velocity : mk(0, 0, 0);
        V3 oB = w->bodies[d.bodyB].angular_velocity;
        const double ve = drive_effective_target(d) - dot(oB - oA, d.axis);
        max_vw = std::max(max_vw, std::fabs(ve));
        if (std::isfinite(d.max_torque)) {
            const double tq = drive_sat_torque(d, drive_deadzone(d, ve));
            if (std::fabs(tq) >= 0.98 * d.max_torque) ++sat;
        }
    }
    w->diag.last_angular_velocity_error = max_vw;
    w->diag.last_torque_saturation_ratio = dc > 0 ? (double)sat / dc : 0.0;
    w->diag.kappa = w->kappa;
    w->diag.dhat = w->dhat;
    w->barrier_form = w->friction_form = w->barrier_in_forms = false;
    const double t6 = now_s();
    w->times[0] = t1 - t0; w->times[1] = t2 - t1; w->times[2] = t3 - t2; w->times[3] = t4 - t3;
    w->times[4] = t5 - t4; w->times[5] = t6 - t0;
}

std::vector<double> vec_from(const double* p, size_t n) { return std::vector<double>(p, p + n); }

}  // namespace

// ===========================================================================
// C API
// ===========================================================================
extern "C" {

void nxd_default_settings(nxd_settings* s);

nxo_world* nxo_create(const nxd_scene_desc* d) {
    if (!d || d->n_bodies < 0) return nullptr;
    auto* w = new nxo_world();
    w->s = d->settings;
    const int N = d->n_bodies;
    // IPCSolver::addAllowedContactPair (IPCSolver.cpp:275-281)
    for (int q = 0; d->contact_pair_bodies && q < d->n_contact_pairs; ++q) {
        const auto key = nxo_world::pair_key(d->contact_pair_bodies[2 * q], d->contact_pair_bodies[2 * q + 1]);
        w->allowed_pairs.insert(key);
        const double f = d->contact_pair_friction ? d->contact_pair_friction[q] : -1.0;
        if (f >= 0.0) w->pair_friction[key] = f;
    }
    w->bodies.resize(N);
    w->meshes.resize(N);
    for (int i = 0; i < N; ++i) {
        Body& b = w->bodies[i];
        b.id = d->body_ids ? d->body_ids[i] : i;
        b.position = getv(d->position, i);
        b.orientation = mkq(d->orientation[4 * i], d->orientation[4 * i + 1], d->orientation[4 * i + 2], d->orientation[4 * i + 3]);
        b.velocity = d->velocity ? getv(d->velocity, i) : mk(0, 0, 0);
        b.angular_velocity = d->angular_velocity ? getv(d->angular_velocity, i) : mk(0, 0, 0);
        b.linear_acceleration = d->linear_acceleration ? getv(d->linear_acceleration, i) : mk(0, 0, 0);
        b.angular_acceleration = d->angular_acceleration ? getv(d->angular_acceleration, i) : mk(0, 0, 0);
        b.mass = d->mass[i];
        for (int k = 0; k < 9; ++k) b.inertia.m[k] = d->inertia_body[9 * i + k];
        Mesh& M = w->meshes[i];
        const int v0 = d->vertex_offset[i], v1 = d->vertex_offset[i + 1];
        const int f0 = d->face_offset[i], f1 = d->face_offset[i + 1];
        if (v1 > v0 && f1 > f0) {
            for (int v = v0; v < v1; ++v) M.V.push_back(getv(d->vertices, v));
            for (int f = f0; f < f1; ++f) M.F.push_back({d->faces[3 * f], d->faces[3 * f + 1], d->faces[3 * f + 2]});
            M.aabb_min = M.V[0]; M.aabb_max = M.V[0];
            for (const auto& p : M.V) { M.aabb_min = cwmin(M.aabb_min, p); M.aabb_max = cwmax(M.aabb_max, p); }
            M.E = build_unique_edges(M.F);
            b.mesh = i;
        }
    }
    for (int j = 0; j < d->n_joints; ++j) {
        Joint J;
        J.type = d->joint_type[j];
        J.bodyA_id = d->joint_body_a[j];
        J.bodyB_id = d->joint_body_b[j];
        const double* p = d->joint_params + (size_t)NXD_JOINT_PARAMS * j;
        switch (J.type) {
            case NXD_JOINT_HINGE:
                J.anchorA = mk(p[0], p[1], p[2]); J.anchorB = mk(p[3], p[4], p[5]);
                J.axisA = mk(p[6], p[7], p[8]); J.axisB = mk(p[9], p[10], p[11]);
                break;
            case NXD_JOINT_SPHERICAL:
                J.anchorA = mk(p[0], p[1], p[2]); J.anchorB = mk(p[3], p[4], p[5]);
                break;
            case NXD_JOINT_FIXED:
                J.target_pos = mk(p[0], p[1], p[2]); J.target_ori = mkq(p[3], p[4], p[5], p[6]);
                break;
            case NXD_JOINT_ANGLE_LIMIT:
                J.axis = normalized(mk(p[0], p[1], p[2])); J.min_angle = p[3]; J.max_angle = p[4];
                break;
            case NXD_JOINT_PRISMATIC:
            case NXD_JOINT_CYLINDRICAL:
                // PrismaticJoint / CylindricalJoint ctors: normalised axes, then
                // JointPrimitives::computeBasis of each
                J.anchorA = mk(p[0], p[1], p[2]); J.anchorB = mk(p[3], p[4], p[5]);
                J.axisA = normalized(mk(p[6], p[7], p[8])); J.axisB = normalized(mk(p[9], p[10], p[11]));
                compute_basis(J.axisA, J.uA, J.vA);
                compute_basis(J.axisB, J.uB, J.vB);
                break;
            case NXD_JOINT_DISTANCE_LIMIT:
                // DistanceLimitJoint ctor (DistanceLimitJoint.cpp:6-15)
                J.min_dist = p[0]; J.max_dist = std::max(p[1], p[0]);
                break;
            default: delete w; return nullptr;
        }
        J.mu = d->joint_stiffness[j];
        J.lambda.assign(J.dim(), 0.0);
        w->joints.push_back(J);
    }
    for (int k = 0; k < d->n_drives; ++k) {
        Drive D;
        const double* p = d->drive_params + (size_t)NXD_DRIVE_PARAMS * k;
        D.kind = d->drive_kind ? d->drive_kind[k] : NXD_DRIVE_ANGULAR_VELOCITY;
        D.bodyA = d->drive_body_a[k] >= 0 ? body_index_of_id(w, d->drive_body_a[k]) : -1;
        D.bodyB = body_index_of_id(w, d->drive_body_b[k]);
        if (D.kind < NXD_DRIVE_ANGULAR_VELOCITY || D.kind > NXD_DRIVE_DAMPED_SPRING || D.bodyB < 0 ||
            D.bodyA == D.bodyB || (D.kind == NXD_DRIVE_DAMPED_SPRING && D.bodyA < 0) ||
            (D.kind == NXD_DRIVE_FORCE && D.bodyA >= 0)) { delete w; return nullptr; }
        if (D.kind == NXD_DRIVE_FORCE) {
            D.force = mk(p[0], p[1], p[2]);
            D.torque = mk(p[3], p[4], p[5]);
        } else if (D.kind == NXD_DRIVE_DAMPED_SPRING) {
            D.rest = p[0]; D.k = p[1]; D.c = p[2];
        } else {
            D.axis = normalized(mk(p[0], p[1], p[2]));
            D.kv = p[3]; D.v_target = p[4];
            D.max_torque = p[5] <= 0.0 ? kInf : p[5];
            D.delay = std::max(0.0, p[6]);
            D.delay_tau = D.kind == NXD_DRIVE_POSITION ? 0.0 : std::max(0.0, p[7]);
        }
        D.filtered = D.v_target;
        w->drives.push_back(D);
    }
    // IPCSolver::setContactDistanceThreshold / setContactStiffness
    w->dhat = std::max(1e-9, w->s.dhat);
    w->kappa = 0.0;
    if (w->s.contact_stiffness > 0.0) w->kappa = w->s.contact_stiffness;
    return w;
}

void nxo_destroy(nxo_world* w) { delete w; }

void nxo_set_options(nxo_world* w, int literal, int stride, int threads) {
    w->literal_min_distance = literal;
    w->md_stride = std::max(1, stride);
    w->num_threads = std::max(1, threads);
}

// Full-IPC time step, restating nxd_ipc_step on the oracle's forms and
// solve: step()'s set-up with the contact forms off, Newton from the
// step-start configuration with the |g|_inf and step (< tol * dt) tests, the rest-form triplets
// followed by the barrier's (the body blocks its active pairs touch, row by
// row), the CCD bound as the first trial of the Armijo search, then step()'s
// write-back.
int nxo_ipc_step(nxo_world* w, double dt, const nxd_ipc_params* p, nxd_ipc_stats* out) {
    const nxd_settings& s = w->s;
    const int N = (int)w->bodies.size(), n = 6 * N;
    std::vector<double> x(n, 0.0), v(n, 0.0), a(n, 0.0);
    for (int i = 0; i < N; ++i) {
        const Body& b = w->bodies[i];
        for (int k = 0; k < 3; ++k) {
            x[i * 6 + k] = b.position[k]; x[i * 6 + 3 + k] = 0.0;
            v[i * 6 + k] = b.velocity[k]; v[i * 6 + 3 + k] = b.angular_velocity[k];
            a[i * 6 + k] = b.linear_acceleration[k]; a[i * 6 + 3 + k] = b.angular_acceleration[k];
        }
    }
    w->x_prev = x; w->v_prev = v; w->a_prev = a; w->dt = dt;
    const bool newmark = s.integrator == NXD_INTEGRATOR_IMPLICIT_NEWMARK;
    const double nm_s1 = (dt * dt) * (0.5 - s.newmark_beta);
    std::vector<double> x_hat(n);
    for (int i = 0; i < n; ++i) {
        x_hat[i] = x[i] + dt * v[i];
        if (newmark) x_hat[i] = x_hat[i] + nm_s1 * a[i];
    }
    w->x_hat = x_hat;
    w->barrier_form = w->friction_form = w->barrier_in_forms = false;
    w->barrier_contacts.clear();
    w->friction_contacts.clear();
    for (auto& d : w->drives) {
        d.dt = dt;
        if (d.delay_tau <= 0.0) { d.filtered = d.v_target; d.filter_init = false; }
        else if (!d.filter_init) { d.filtered = d.v_target; d.filter_init = true; }
        else if (d.dt > 0.0) { const double al = d.dt / (d.delay_tau + d.dt); d.filtered += al * (d.v_target - d.filtered); }
        d.gA = d.bodyA >= 0 ? d.bodyA * 6 : -1;
        d.gB = d.bodyB >= 0 ? d.bodyB * 6 : -1;
        d.has_prev = false;
    }
    for (auto& J : w->joints) {
        const int ia = body_index_of_id(w, J.bodyA_id);
        if (J.type == NXD_JOINT_FIXED) {
            J.gA = ia * 6; J.qA_ref = w->bodies[ia].orientation;
        } else {
            const int ib = body_index_of_id(w, J.bodyB_id);
            J.gA = ia * 6; J.gB = ib * 6;
            J.pA_ref = w->bodies[ia].position; J.qA_ref = w->bodies[ia].orientation;
            J.pB_ref = w->bodies[ib].position; J.qB_ref = w->bodies[ib].orientation;
        }
    }
    const double sc = scaling(w);
    std::vector<double> xn = x, gr, gb(n), g(n), Hb((size_t)n * n), dx, xt(n), prod(n);
    std::vector<Trip> trips;
    std::vector<std::pair<int, int>> blocks;
    int iters = 0, conv = 0, lsfail = 0, solvefail = 0, iters_done = 0;
    int64_t npairs = 0, na = 0, nfric = 0;
    double amax = 1.0, fx = 0.0;
    // lagged friction: pass 0 freezes the pairs active at the step start,
    // each further pass those at the previous pass's solution
    const bool friction = p->mu > 0.0;
    const int passes = friction ? p->friction_iters : 1;
    IpcFricCtx* fr = friction ? ipc_fric_new(p->mu, p->friction_eps) : nullptr;
    for (int pass = 0; pass < passes; ++pass) {
        if (fr) ipc_fric_rebuild(fr);
        conv = 0;
        iters = 0;
        for (int it = 0; it < p->newton_max_iters; ++it) {
            iters = it;
            problem_gradient(w, xn, gr);
            double eb = 0.0;
            blocks.clear();
            ipc_barrier_cpu(w, xn.data(), p->dhat, p->kappa, &eb, gb.data(), Hb.data(), &blocks, &npairs, &na, fr);
            if (fr) { eb = eb + ipc_fric_energy(fr); nfric = ipc_fric_count(fr); }
            for (int i = 0; i < n; ++i) g[i] = gr[i] + sc * gb[i];
            double ginf = 0.0;
            for (double vv : g) ginf = std::max(ginf, std::fabs(vv));
            if (ginf < p->newton_tol) { conv = 1; break; }
            problem_hessian(w, xn, trips);
            for (const auto& bl : blocks)
                for (int r = 0; r < 6; ++r)
                    for (int c = 0; c < 6; ++c) {
                        const int gi = 6 * bl.first + r, gj = 6 * bl.second + c;
                        trips.push_back({gi, gj, Hb[(size_t)gi * n + gj] * sc});
                    }
            std::vector<double> rhs(n);
            for (int i = 0; i < n; ++i) rhs[i] = -g[i];
            if (!solve_system(n, trips, rhs, dx)) { solvefail = 1; break; }
            double dxinf = 0.0;
            for (double vv : dx) dxinf = std::max(dxinf, std::fabs(vv));
            if (dxinf < p->newton_tol * dt) { conv = 1; break; }
            int64_t np2 = 0;
            amax = nxo_ipc_max_step(w, xn.data(), dx.data(), p->eta, &np2);
            fx = problem_value(w, xn) + sc * eb;
            for (int i = 0; i < n; ++i) prod[i] = g[i] * dx[i];
            const double descent = tree_sum(prod);
            if (descent > 0) { lsfail = 1; break; }
            double alpha = std::min(1.0, amax);
            bool done = false;
            for (int ls = 0; ls < p->ls_max_iters; ++ls) {
                for (int i = 0; i < n; ++i) xt[i] = xn[i] + alpha * dx[i];
                const double ert = problem_value(w, xt);
                double ebt = 0.0;
                ipc_barrier_cpu(w, xt.data(), p->dhat, p->kappa, &ebt, nullptr, nullptr, nullptr, nullptr, nullptr, fr);
                if (fr) ebt = ebt + ipc_fric_energy(fr);
                const double fn = ert + sc * ebt;
                if (fn <= fx + s.ls_c1 * alpha * descent) { done = true; fx = fn; break; }
                alpha *= s.ls_rho;
            }
            if (!done) { lsfail = 1; break; }
            xn = xt;
            if (it == p->newton_max_iters - 1) iters = p->newton_max_iters;
        }
        iters_done += iters;
        if (!conv) break;   // a pass that did not converge ends the step
    }
    iters = iters_done;
    if (fr) ipc_fric_free(fr);
    std::vector<double> vn(n), an(n);
    if (newmark) {
        const double den = (s.newmark_beta * dt) * dt;
        for (int i = 0; i < n; ++i) an[i] = (xn[i] - w->x_hat[i]) / den;
        for (int i = 0; i < n; ++i)
            vn[i] = w->v_prev[i] + dt * ((1.0 - s.newmark_gamma) * w->a_prev[i] + s.newmark_gamma * an[i]);
    } else {
        for (int i = 0; i < n; ++i) vn[i] = (xn[i] - w->x_prev[i]) / dt;
        for (int i = 0; i < n; ++i) an[i] = (vn[i] - w->v_prev[i]) / dt;
    }
    for (int i = 0; i < N; ++i) {
        Body& b = w->bodies[i];
        const int idx = i * 6;
        b.linear_acceleration = xseg(an, idx);
        b.angular_acceleration = xseg(an, idx + 3);
        b.velocity = xseg(vn, idx);
        b.angular_velocity = xseg(vn, idx + 3);
        b.position = xseg(xn, idx);
        b.orientation = update_rotation_gt(b.orientation, xseg(xn, idx + 3));
    }
    if (out) {
        out->newton_iterations = iters; out->converged = conv; out->line_search_failed = lsfail;
        out->solve_failed = solvefail; out->last_alpha_max = amax; out->energy = fx; out->n_pairs = npairs;
        out->n_active = na; out->pcg_iterations = 0; out->n_friction = nfric;
    }
    return solvefail ? NXD_FACTOR_FAILED : NXD_OK;
}

int nxo_step(nxo_world* w, double dt) {
    step(w, dt);
    return NXD_OK;
}

int nxo_get_state(nxo_world* w, const nxd_state* o) {
    for (int i = 0; i < (int)w->bodies.size(); ++i) {
        const Body& b = w->bodies[i];
        if (o->position) setv(o->position, i, b.position);
        if (o->orientation) { o->orientation[4 * i] = b.orientation.w; o->orientation[4 * i + 1] = b.orientation.x;
                              o->orientation[4 * i + 2] = b.orientation.y; o->orientation[4 * i + 3] = b.orientation.z; }
        if (o->velocity) setv(o->velocity, i, b.velocity);
        if (o->angular_velocity) setv(o->angular_velocity, i, b.angular_velocity);
        if (o->linear_acceleration) setv(o->linear_acceleration, i, b.linear_acceleration);
        if (o->angular_acceleration) setv(o->angular_acceleration, i, b.angular_acceleration);
    }
    return NXD_OK;
}
int nxo_set_state(nxo_world* w, const nxd_state* o) {
    for (int i = 0; i < (int)w->bodies.size(); ++i) {
        Body& b = w->bodies[i];
        if (o->position) b.position = getv(o->position, i);
        if (o->orientation) b.orientation = mkq(o->orientation[4 * i], o->orientation[4 * i + 1], o->orientation[4 * i + 2], o->orientation[4 * i + 3]);
        if (o->velocity) b.velocity = getv(o->velocity, i);
        if (o->angular_velocity) b.angular_velocity = getv(o->angular_velocity, i);
        if (o->linear_acceleration) b.linear_acceleration = getv(o->linear_acceleration, i);
        if (o->angular_acceleration) b.angular_acceleration = getv(o->angular_acceleration, i);
    }
    return NXD_OK;
}
int nxo_get_diagnostics(nxo_world* w, nxd_diagnostics* o) {
    *o = w->diag;
    o->kappa = w->kappa;
    o->dhat = w->dhat;
    return NXD_OK;
}
int nxo_get_joint_state(nxo_world* w, double* lam, double* stiff) {
    for (size_t j = 0; j < w->joints.size(); ++j) {
        for (int k = 0; k < 6; ++k) if (lam) lam[6 * j + k] = k < (int)w->joints[j].lambda.size() ? w->joints[j].lambda[k] : 0.0;
        if (stiff) stiff[j] = w->joints[j].mu;
    }
    return NXD_OK;
}
void nxo_last_step_times(nxo_world* w, double* o) { for (int i = 0; i < 6; ++i) o[i] = w->times[i]; }

int64_t nxo_body_pairs(nxo_world* w, double r, int32_t* pairs, int64_t cap) {
    assembler_build(w);
    const auto p = detect_body_pairs(w, r);
    for (int64_t i = 0; i < (int64_t)p.size() && i < cap; ++i) { pairs[2 * i] = p[i].first; pairs[2 * i + 1] = p[i].second; }
    return (int64_t)p.size();
}

int nxo_build_candidates(nxo_world* w, double act, nxd_candidates* o) {
    assembler_build(w);
    Candidates c;
    build_candidate_set(w, act, c);
    int st = NXD_OK;
    auto put = [&](int32_t* buf, int64_t cap, int64_t& count, size_t n, int width, auto&& fill) {
        count = (int64_t)n;
        if (!buf) return;
        if ((int64_t)n > cap) st = NXD_CAPACITY;
        for (size_t i = 0; i < n && (int64_t)i < cap; ++i) fill(buf + width * i, i);
    };
    put(o->vv, o->vv_cap, o->vv_count, c.vv.size(), 4, [&](int32_t* r, size_t i) { r[0] = c.vv[i].b0; r[1] = c.vv[i].b1; r[2] = c.vv[i].v0; r[3] = c.vv[i].v1; });
    put(o->ev, o->ev_cap, o->ev_count, c.ev.size(), 5, [&](int32_t* r, size_t i) { r[0] = c.ev[i].eb; r[1] = c.ev[i].vb; r[2] = c.ev[i].e0; r[3] = c.ev[i].e1; r[4] = c.ev[i].v; });
    put(o->ee, o->ee_cap, o->ee_count, c.ee.size(), 6, [&](int32_t* r, size_t i) { r[0] = c.ee[i].b0; r[1] = c.ee[i].b1; r[2] = c.ee[i].a0; r[3] = c.ee[i].a1; r[4] = c.ee[i].c0; r[5] = c.ee[i].c1; });
    put(o->fv, o->fv_cap, o->fv_count, c.fv.size(), 4, [&](int32_t* r, size_t i) { r[0] = c.fv[i].fb; r[1] = c.fv[i].vb; r[2] = c.fv[i].f; r[3] = c.fv[i].v; });
    return st;
}

int nxo_detect_contacts(nxo_world* w, const double* x, nxd_contact* out, int32_t cap, int32_t* count, int32_t* raw_count) {
    assembler_build(w);
    build_candidate_set(w, w->dhat, w->cand);
    std::vector<double> xv;
    if (x) xv = vec_from(x, w->bodies.size() * 6);
    int raw = 0;
    const auto cs = detect_contacts(w, x ? &xv : nullptr, &raw);
    if (count) *count = (int32_t)cs.size();
    if (raw_count) *raw_count = raw;
    for (size_t i = 0; i < cs.size() && (int32_t)i < cap; ++i) {
        nxd_contact& c = out[i];
        for (int k = 0; k < 3; ++k) { c.point[k] = cs[i].point[k]; c.normal[k] = cs[i].normal[k]; }
        c.distance = cs[i].distance;
        c.body_a = cs[i].bodyA; c.body_b = cs[i].bodyB; c.primitive_type = cs[i].type;
        c.primitive_a = cs[i].primA; c.primitive_b = cs[i].primB; c.pad_ = 0;
    }
    return (int32_t)cs.size() > cap ? NXD_CAPACITY : NXD_OK;
}

double nxo_scene_min_distance(nxo_world* w, int literal) {
    return literal ? scene_min_distance_literal(w) : scene_min_distance_pruned(w);
}

double nxo_max_step(nxo_world* w, double dt) {
    assembler_build(w);
    build_candidate_set(w, w->dhat, w->cand);
    return compute_max_step(w, dt);
}

int nxo_set_form_state(nxo_world* w, const nxd_contact* cs, int32_t n, const double* nf, const double* xh, double dt) {
    w->barrier_contacts.clear();
    for (int i = 0; i < n; ++i) {
        Contact c;
        c.bodyA = cs[i].body_a; c.bodyB = cs[i].body_b; c.type = cs[i].primitive_type;
        c.primA = cs[i].primitive_a; c.primB = cs[i].primitive_b;
        c.point = mk(cs[i].point[0], cs[i].point[1], cs[i].point[2]);
        c.normal = mk(cs[i].normal[0], cs[i].normal[1], cs[i].normal[2]);
        c.distance = cs[i].distance;
        w->barrier_contacts.push_back(c);
    }
    w->friction_contacts = w->barrier_contacts;
    w->normal_forces.clear();
    if (nf) w->normal_forces.assign(nf, nf + n);
    if (xh) w->x_hat = vec_from(xh, w->bodies.size() * 6);
    else if (w->x_hat.size() != w->bodies.size() * 6) w->x_hat.assign(w->bodies.size() * 6, 0.0);
    w->dt = dt;
    w->friction_dt = std::max(0.0, dt);
    w->barrier_dhat = std::max(1e-9, w->dhat);
    w->barrier_kappa = std::max(0.0, w->kappa);
    w->friction_mu = w->s.friction_coeff;
    w->friction_eps = 1e-8;
    w->barrier_form = true;
    w->barrier_in_forms = w->s.enable_adaptive_barrier != 0;
    w->friction_form = w->s.enable_friction && w->s.friction_coeff > 0;
    for (auto& J : w->joints) {
        const int ia = body_index_of_id(w, J.bodyA_id);
        if (J.type == NXD_JOINT_FIXED) { J.gA = ia * 6; J.qA_ref = w->bodies[ia].orientation; }
        else {
            const int ib = body_index_of_id(w, J.bodyB_id);
            J.gA = ia * 6; J.gB = ib * 6;
            J.pA_ref = w->bodies[ia].position; J.qA_ref = w->bodies[ia].orientation;
            J.pB_ref = w->bodies[ib].position; J.qB_ref = w->bodies[ib].orientation;
        }
    }
    for (auto& d : w->drives) {
        d.dt = dt; d.gA = d.bodyA >= 0 ? d.bodyA * 6 : -1; d.gB = d.bodyB >= 0 ? d.bodyB * 6 : -1; d.has_prev = false;
    }
    return NXD_OK;
}

int nxo_form_value(nxo_world* w, int32_t form, const double* xp, double* out) {
    const auto x = vec_from(xp, w->bodies.size() * 6);
    switch (form) {
        case NXD_FORM_INERTIA: *out = inertia_value(w, x); break;
        case NXD_FORM_GRAVITY: *out = gravity_value(w, x); break;
        case NXD_FORM_CONSTRAINT: *out = constraint_value(w, x); break;
        case NXD_FORM_BARRIER: *out = barrier_form_value(w, x); break;
        case NXD_FORM_FRICTION: *out = friction_form_value(w, x); break;
        case NXD_FORM_DRIVES: *out = drives_value(w, x); break;
        case NXD_FORM_TOTAL: *out = problem_value(w, x); break;
        case NXD_FORM_CONTACT: *out = problem_contact_value(w, x); break;
        default: return NXD_INVALID_ARGUMENT;
    }
    return NXD_OK;
}

int nxo_form_gradient(nxo_world* w, int32_t form, const double* xp, double* gp) {
    const size_t n = w->bodies.size() * 6;
    const auto x = vec_from(xp, n);
    std::vector<double> g(n, 0.0);
    switch (form) {
        case NXD_FORM_INERTIA: inertia_gradient(w, x, g); break;
        case NXD_FORM_GRAVITY: gravity_gradient(w, g); break;
        case NXD_FORM_CONSTRAINT: for (const auto& J : w->joints) joint_gradient(J, x, g); break;
        case NXD_FORM_BARRIER: barrier_form_gradient(w, x, g); break;
        case NXD_FORM_FRICTION: friction_form_gradient(w, x, g); break;
        case NXD_FORM_DRIVES: for (auto& d : w->drives) drive_gradient(w, d, x, g); break;
        case NXD_FORM_TOTAL: problem_gradient(w, x, g); break;
        case NXD_FORM_CONTACT: problem_contact_gradient(w, x, g); break;
        default: return NXD_INVALID_ARGUMENT;
    }
    std::copy(g.begin(), g.end(), gp);
    return NXD_OK;
}

int nxo_form_hessian_dense(nxo_world* w, int32_t form, const double* xp, double* H) {
    const size_t n = w->bodies.size() * 6;
    const auto x = vec_from(xp, n);
    std::vector<Trip> t;
    const double s = scaling(w);
    switch (form) {
        case NXD_FORM_INERTIA: inertia_hessian(w, t); break;
        case NXD_FORM_GRAVITY: break;
        case NXD_FORM_CONSTRAINT: for (const auto& J : w->joints) joint_hessian(J, x, t); break;
        case NXD_FORM_BARRIER: barrier_form_hessian(w, x, t); break;
        case NXD_FORM_FRICTION: friction_form_hessian(w, x, t); break;
        case NXD_FORM_DRIVES: for (auto& d : w->drives) drive_hessian(d, x, t); break;
        case NXD_FORM_TOTAL: problem_hessian(w, x, t); break;
        case NXD_FORM_CONTACT: {
            std::vector<Trip> tt;
            if (w->barrier_in_forms) { barrier_form_hessian(w, x, tt); for (auto& q : tt) t.push_back({q.r, q.c, q.v * s}); }
            tt.clear();
            if (w->friction_form) { friction_form_hessian(w, x, tt); for (auto& q : tt) t.push_back({q.r, q.c, q.v * s}); }
            break;
        }
        default: return NXD_INVALID_ARGUMENT;
    }
    std::fill(H, H + n * n, 0.0);
    for (const auto& q : t) H[(size_t)q.r * n + q.c] += q.v;
    return NXD_OK;
}

int nxo_linear_solve(int32_t n_rows, int64_t nnzb, const int32_t* row_ptr, const int32_t* col_idx,
                     const double* vals, const double* b, double* x) {
    std::vector<Trip> trips;
    trips.reserve((size_t)nnzb * 36);
    for (int i = 0; i < n_rows; ++i)
        for (int64_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k)
            for (int r = 0; r < 6; ++r)
                for (int cc = 0; cc < 6; ++cc) trips.push_back({6 * i + r, 6 * col_idx[k] + cc, vals[36 * k + 6 * r + cc]});
    const int n = 6 * n_rows;
    std::vector<double> rhs(b, b + n), sol;
    if (!solve_system(n, trips, rhs, sol)) return NXD_FACTOR_FAILED;
    for (int i = 0; i < n; ++i) x[i] = sol[i];
    return NXD_OK;
}

int nxo_normal_forces(nxo_world* w, const double* xp, double* out, int32_t n) {
    const auto x = vec_from(xp, w->bodies.size() * 6);
    const auto nf = barrier_normal_forces(w, x);
    for (int i = 0; i < n && i < (int)nf.size(); ++i) out[i] = nf[i];
    return NXD_OK;
}

int nxo_ldlt_solve(const double* H, int32_t n, const double* b, double* x) {
    std::vector<Trip> t;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            if (H[(size_t)i * n + j] != 0.0) t.push_back({i, j, H[(size_t)i * n + j]});
    std::vector<double> rhs(b, b + n), sol;
    if (!solve_system(n, t, rhs, sol)) return NXD_FACTOR_FAILED;
    std::copy(sol.begin(), sol.end(), x);
    return NXD_OK;
}

void nxo_libm(int32_t fn, const double* x, const double* y, double* out, int32_t n) {
    for (int i = 0; i < n; ++i) {
        switch (fn) {
            case 0: out[i] = nxm::sin(x[i]); break;
            case 1: out[i] = nxm::cos(x[i]); break;
            case 2: out[i] = nxm::atan2(x[i], y[i]); break;
            case 3: out[i] = nxm::log(x[i]); break;
            case 4: out[i] = nxm::exp(x[i]); break;
            case 5: out[i] = nxm::tanh(x[i]); break;
            default: out[i] = nxm::cosh(x[i]); break;
        }
    }
}

void nxo_select_top_k(const double* scores, int32_t n, int32_t k, int32_t* out) {
    const auto idx = select_top_k_indices(n, k, [&](int i) { return scores[i]; });
    for (size_t i = 0; i < idx.size(); ++i) out[i] = idx[i];
}
void nxo_std_sort(const double* keys, int32_t n, int32_t* idx) {
    std::sort(idx, idx + n, [&](int a, int b) { return keys[a] < keys[b]; });
}

double nxo_barrier_value(double d, double dh, double k) { return barrier_value(d, dh, k); }
double nxo_barrier_gradient(double d, double dh, double k) { return barrier_gradient(d, dh, k); }
double nxo_barrier_hessian(double d, double dh, double k) { return barrier_hessian(d, dh, k); }
double nxo_friction_value(const double* u, double N, double mu, double eps) { return fric_value(mk(u[0], u[1], u[2]), N, mu, eps); }
void nxo_friction_gradient(const double* u, double N, double mu, double eps, double* g) {
    const V3 r = fric_gradient(mk(u[0], u[1], u[2]), N, mu, eps); g[0] = r.x; g[1] = r.y; g[2] = r.z;
}
void nxo_friction_hessian(const double* u, double N, double mu, double eps, double* H) {
    const M3 r = fric_hessian(mk(u[0], u[1], u[2]), N, mu, eps); for (int i = 0; i < 9; ++i) H[i] = r.m[i];
}
// FrictionPotential::*Smooth (src/Physics/Contact/Friction.cpp:63-132)
double nxo_friction_value_smooth(const double* u, double N, double mu, double eps) {
    if (N <= 0) return 0.0;
    const double un = norm(mk(u[0], u[1], u[2]));
    if (un <= eps) return 0.5 * mu * N / eps * un * un;
    return mu * N * (un - 0.5 * eps);
}
void nxo_friction_gradient_smooth(const double* u, double N, double mu, double eps, double* g) {
    g[0] = g[1] = g[2] = 0.0;
    if (N <= 0) return;
    const V3 uu = mk(u[0], u[1], u[2]);
    const double un = norm(uu);
    if (un < 1e-12) return;
    const V3 uh = uu / un;
    const V3 r = un <= eps ? mu * N / eps * uu : mu * N * uh;
    g[0] = r.x; g[1] = r.y; g[2] = r.z;
}
void nxo_friction_hessian_smooth(const double* u, double N, double mu, double eps, double* H) {
    for (int i = 0; i < 9; ++i) H[i] = 0.0;
    if (N <= 0) return;
    const V3 uu = mk(u[0], u[1], u[2]);
    const double un = norm(uu);
    if (un < 1e-12 || un <= eps) { for (int i = 0; i < 3; ++i) H[4 * i] = mu * N / eps; return; }
    const V3 uh = uu / un;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) H[3 * i + j] = (mu * N / un) * ((i == j ? 1.0 : 0.0) - uh[i] * uh[j]);
}

// 1-D intervalRootFinder (IntervalRootFinder.h:163-190 -> 20-114) on a polynomial.
int nxo_interval_root_poly(const double* c, int32_t deg, double lo, double hi, double tol, double* rlo, double* rhi) {
    auto f = [&](Ivl x) {
        Ivl acc = iv(c[deg]);
        for (int k = deg - 1; k >= 0; --k) acc = acc * x + iv(c[k]);
        return acc;
    };
    Ivl earliest = iv(kInf);
    bool found = false;
    std::stack<Ivl> xs;
    xs.push(iv(lo, hi));
    for (int it = 0; !xs.empty() && it < 1000; ++it) {
        Ivl x = xs.top(); xs.pop();
        if (x.lo >= earliest.lo) continue;
        Ivl y = f(x);
        if (!zero_in(y)) continue;
        if (x.hi - x.lo <= tol) {
            if (x.lo < earliest.lo) { earliest = x; found = true; }
            continue;
        }
        const double mid = 0.5 * (x.lo + x.hi);
        xs.push(iv(x.lo, mid));
        xs.push(iv(mid, x.hi));
    }
    if (found) { *rlo = earliest.lo; *rhi = earliest.hi; }
    return found ? 1 : 0;
}

// ---------------------------------------------------------------------------
// Geometry accessors for the primitive-level (full IPC) checker in
// ipc_cpu.cpp: primitives numbered over bodies in world order (vertices,
// faces, unique edges of each body's mesh; meshless bodies have none), the
// same numbering the device uses.
// ---------------------------------------------------------------------------
int32_t nxo_body_count(nxo_world* w) { return (int32_t)w->bodies.size(); }

void nxo_prim_counts(nxo_world* w, int64_t* nv, int64_t* nf, int64_t* ne) {
    int64_t a = 0, b = 0, c = 0;
    for (const Body& B : w->bodies) {
        if (B.mesh < 0) continue;
        const Mesh& M = w->meshes[B.mesh];
        a += (int64_t)M.V.size(); b += (int64_t)M.F.size(); c += (int64_t)M.E.size();
    }
    *nv = a; *nf = b; *ne = c;
}

void nxo_prim_topology(nxo_world* w, int32_t* vbody, int32_t* fbody, int32_t* fvert, int32_t* ebody, int32_t* evert) {
    int vo = 0, fo = 0, eo = 0;
    for (int i = 0; i < (int)w->bodies.size(); ++i) {
        const Body& B = w->bodies[i];
        if (B.mesh < 0) continue;
        const Mesh& M = w->meshes[B.mesh];
        for (size_t v = 0; v < M.V.size(); ++v) vbody[vo + v] = i;
        for (size_t f = 0; f < M.F.size(); ++f) {
            fbody[fo + f] = i;
            for (int k = 0; k < 3; ++k) fvert[3 * (fo + f) + k] = vo + M.F[f][k];
        }
        for (size_t e = 0; e < M.E.size(); ++e) {
            ebody[eo + e] = i;
            for (int k = 0; k < 2; ++k) evert[2 * (eo + e) + k] = vo + M.E[e][k];
        }
        vo += (int)M.V.size(); fo += (int)M.F.size(); eo += (int)M.E.size();
    }
}

// World vertices and body positions at state x (6N; p = x[6i..], q =
// exp(theta) q_body as in detectContactsAtState), or at the current poses
// when x is NULL.
// Body-local vertex coordinates in the global numbering (bodies in order)
// and each body's orientation (w, x, y, z): the arc motion of the CCD.
void nxo_local_vertices(nxo_world* w, double* vloc, double* quat) {
    int vo = 0;
    for (int i = 0; i < (int)w->bodies.size(); ++i) {
        const Body& B = w->bodies[i];
        if (quat) { quat[4 * i] = B.orientation.w; quat[4 * i + 1] = B.orientation.x; quat[4 * i + 2] = B.orientation.y; quat[4 * i + 3] = B.orientation.z; }
        if (B.mesh < 0) continue;
        const Mesh& M = w->meshes[B.mesh];
        for (size_t v = 0; v < M.V.size(); ++v) {
            if (vloc) { vloc[3 * (vo + v)] = M.V[v].x; vloc[3 * (vo + v) + 1] = M.V[v].y; vloc[3 * (vo + v) + 2] = M.V[v].z; }
        }
        vo += (int)M.V.size();
    }
}

void nxo_world_vertices_at(nxo_world* w, const double* x, double* wv, double* pos) {
    int vo = 0;
    for (int i = 0; i < (int)w->bodies.size(); ++i) {
        const Body& B = w->bodies[i];
        V3 p = B.position;
        Q q = B.orientation;
        if (x) {
            p = V3{x[6 * i], x[6 * i + 1], x[6 * i + 2]};
            q = update_rotation_gt(B.orientation, V3{x[6 * i + 3], x[6 * i + 4], x[6 * i + 5]});
        }
        if (pos) { pos[3 * i] = p.x; pos[3 * i + 1] = p.y; pos[3 * i + 2] = p.z; }
        if (B.mesh < 0) continue;
        const Mesh& M = w->meshes[B.mesh];
        for (size_t v = 0; v < M.V.size(); ++v) {
            const V3 a = p + qrot(q, M.V[v]);
            wv[3 * (vo + v)] = a.x; wv[3 * (vo + v) + 1] = a.y; wv[3 * (vo + v) + 2] = a.z;
        }
        vo += (int)M.V.size();
    }
}

}  // extern "C"
