// phx_csg.cuh : ray intersection with one CSG prim (a complete binary tree of CSGNode).
//
// Semantics follow the reference's IS path:
//   intersect_prim  CSG/csg_intersect_tree.h:684-719
//   intersect_tree  CSG/csg_intersect_tree.h:277-672  (Kensler single-hit CSG over a postorder
//                   walk of the complete tree, re-walking sub-trees from an advanced tmin)
//   intersect_leaf  CSG/csg_intersect_leaf.h:175-300  (node transform, normal back-transform,
//                   complement signalled by the sign of isect.x)
//   leaves          sphere  CSG/csg_intersect_leaf_sphere.h:15-40
//                   zsphere CSG/csg_intersect_leaf_zsphere.h:45-153
//                   cylinder CSG/csg_intersect_leaf_cylinder.h:34-95
//                   box3    CSG/csg_intersect_leaf_box3.h:64-157
//                   roots   CSG/csg_robust_quadratic_roots.h:95-122
// The torus leaf has no counterpart in the current reference intersector; it is a new FP64
// quartic solve (monotone-interval Newton/bisection) written for this engine.
//
// The node table is read through the read-only data path; nodes are 64 B (4 x float4).
#pragma once
#include "phx_vec.cuh"
#include "phx_pod.h"

#define PHX_CSG_STACK 15
#define PHX_TRANCHE_STACK 4
#define PHX_CSG_PROPAGATE_EPSILON 0.0001f

enum { PHX_CSG_ERR_OVERFLOW = 1, PHX_CSG_ERR_POP_EMPTY = 2, PHX_CSG_ERR_XOR_SIDE = 4,
       PHX_CSG_ERR_END_EMPTY = 8, PHX_CSG_ERR_TRANCHE = 16 };

enum { PHX_STATE_ENTER = 0, PHX_STATE_EXIT = 1, PHX_STATE_MISS = 2 };
enum { PHX_CTRL_RETURN_MISS = 0, PHX_CTRL_RETURN_A = 1, PHX_CTRL_RETURN_B = 2,
       PHX_CTRL_RETURN_FLIP_B = 3, PHX_CTRL_LOOP_A = 4, PHX_CTRL_LOOP_B = 5 };

// Kensler's single-hit boolean action table, resolved for "A closer" and "B closer".
// Each operation maps (stateA, stateB) to an action; the eight non-miss/miss pairs are
// packed four bits each at offset 3*stateA+stateB.  The values are generated from the rules
// of the paper in phx_csg_ctrl() below and checked against this packing on the host.
struct PhxCsgRules {
    // returns the action for op in {1:union,2:intersection,3:difference}
    static __host__ __device__ constexpr int ctrl(int op, int a, int b, bool aCloser)
    {
        // union
        return op == PHX_CSG_UNION ? (
                   a == PHX_STATE_ENTER && b == PHX_STATE_ENTER ? (aCloser ? PHX_CTRL_RETURN_A : PHX_CTRL_RETURN_B) :
                   a == PHX_STATE_ENTER && b == PHX_STATE_EXIT  ? (aCloser ? PHX_CTRL_LOOP_A : PHX_CTRL_RETURN_B) :
                   a == PHX_STATE_EXIT  && b == PHX_STATE_ENTER ? (aCloser ? PHX_CTRL_RETURN_A : PHX_CTRL_LOOP_B) :
                   a == PHX_STATE_EXIT  && b == PHX_STATE_EXIT  ? (aCloser ? PHX_CTRL_RETURN_B : PHX_CTRL_RETURN_A) :
                   a == PHX_STATE_MISS  && b == PHX_STATE_MISS  ? PHX_CTRL_RETURN_MISS :
                   b == PHX_STATE_MISS ? PHX_CTRL_RETURN_A : PHX_CTRL_RETURN_B )
             : op == PHX_CSG_INTERSECTION ? (
                   a == PHX_STATE_MISS || b == PHX_STATE_MISS ? PHX_CTRL_RETURN_MISS :
                   a == PHX_STATE_ENTER && b == PHX_STATE_ENTER ? (aCloser ? PHX_CTRL_LOOP_A : PHX_CTRL_LOOP_B) :
                   a == PHX_STATE_ENTER && b == PHX_STATE_EXIT  ? (aCloser ? PHX_CTRL_RETURN_A : PHX_CTRL_LOOP_B) :
                   a == PHX_STATE_EXIT  && b == PHX_STATE_ENTER ? (aCloser ? PHX_CTRL_LOOP_A : PHX_CTRL_RETURN_B) :
                   (aCloser ? PHX_CTRL_RETURN_A : PHX_CTRL_RETURN_B) )
             : /* difference A - B */ (
                   a == PHX_STATE_MISS ? PHX_CTRL_RETURN_MISS :
                   b == PHX_STATE_MISS ? PHX_CTRL_RETURN_A :
                   a == PHX_STATE_ENTER && b == PHX_STATE_ENTER ? (aCloser ? PHX_CTRL_RETURN_A : PHX_CTRL_LOOP_B) :
                   a == PHX_STATE_ENTER && b == PHX_STATE_EXIT  ? (aCloser ? PHX_CTRL_LOOP_A : PHX_CTRL_LOOP_B) :
                   a == PHX_STATE_EXIT  && b == PHX_STATE_ENTER ? (aCloser ? PHX_CTRL_RETURN_A : PHX_CTRL_RETURN_FLIP_B) :
                   (aCloser ? PHX_CTRL_LOOP_A : PHX_CTRL_RETURN_FLIP_B) );
    }
    static __host__ __device__ constexpr unsigned packed(int op, bool aCloser)
    {
        return  (unsigned)ctrl(op, 0, 0, aCloser)       | (unsigned)ctrl(op, 0, 1, aCloser) << 4
              | (unsigned)ctrl(op, 0, 2, aCloser) << 8  | (unsigned)ctrl(op, 1, 0, aCloser) << 12
              | (unsigned)ctrl(op, 1, 1, aCloser) << 16 | (unsigned)ctrl(op, 1, 2, aCloser) << 20
              | (unsigned)ctrl(op, 2, 0, aCloser) << 24 | (unsigned)ctrl(op, 2, 1, aCloser) << 28;
    }
};

PHX_D int phx_csg_lookup(int op, int sa, int sb, bool aCloser)
{
    // the packed words are compile-time constants; one shift+mask per combine
    const unsigned wA = op == PHX_CSG_UNION ? PhxCsgRules::packed(1, true)
                      : op == PHX_CSG_INTERSECTION ? PhxCsgRules::packed(2, true) : PhxCsgRules::packed(3, true);
    const unsigned wB = op == PHX_CSG_UNION ? PhxCsgRules::packed(1, false)
                      : op == PHX_CSG_INTERSECTION ? PhxCsgRules::packed(2, false) : PhxCsgRules::packed(3, false);
    const unsigned w = aCloser ? wA : wB;
    const unsigned off = 3u * (unsigned)sa + (unsigned)sb;
    return off < 8u ? (int)((w >> (off * 4u)) & 0xfu) : PHX_CTRL_RETURN_MISS;
}

struct PhxCsgCtx {
    const float4* node;   // (Nn*4) float4 : CSGNode table
    const float4* itra;   // (Nt*4) float4 : inverse node transforms
    const float4* plan;   // (Nl) float4 : planes of convex polyhedra (n, w)
};

// CSG evaluator variant, the template argument of the trace chain: bit 0 the FP64 root polish,
// bit 1 the full evaluator (the leaves beyond sphere, zsphere, cylinder, box3 and torus, and list
// nodes).  The host launches the full variant only for geometries that use it: in the base
// variant the leaf dispatch and tree walk keep the registers and code size of those five leaves.
#define PHX_CV_POLISH 1
#define PHX_CV_FULL 2
#define PHX_CV_P(cv) (((cv) & PHX_CV_POLISH) != 0)
#define PHX_CV_F(cv) (((cv) & PHX_CV_FULL) != 0)

// typecodes the base variant evaluates (operators, CSG_ZERO and the five leaves)
__host__ __device__ inline bool phx_csg_base_typecode(unsigned tc)
{
    return tc <= 3u || tc == 101u || tc == 103u || tc == 105u || tc == 110u || tc == 116u;
}

PHX_D unsigned nd_u(const float4& q, int k) { return __float_as_uint(k == 0 ? q.x : k == 1 ? q.y : k == 2 ? q.z : q.w); }

// ---------------------------------------------------------------- quadratic roots
// Solve d t^2 + 2 b t + c = 0 choosing the form of each root that avoids cancellation.
PHX_D void robust_roots(float& t1, float& t2, float& disc, float& sdisc, const float d, const float b, const float c)
{
    disc = b * b - d * c;
    sdisc = disc > 0.f ? sqrtf(disc) : 0.f;
    float q = b > 0.f ? -(b + sdisc) : -(b - sdisc);
    float root1 = q / d;
    float root2 = c / q;
    t1 = fminf(root1, root2);
    t2 = fmaxf(root1, root2);
}
PHX_D void robust_roots_disq(const float t_min, float& t1, float& t2, float& disc, float& sdisc, const float d, const float b, const float c)
{
    disc = b * b - d * c;
    sdisc = disc > 0.f ? sqrtf(disc) : 0.f;
    float q = b > 0.f ? -(b + sdisc) : -(b - sdisc);
    float root1 = sdisc > 0.f ? q / d : t_min;
    float root2 = sdisc > 0.f ? c / q : t_min;
    t1 = fminf(root1, root2);
    t2 = fmaxf(root1, root2);
}
// FP64 re-solve of the same quadratic from the same (FP32) ray and shape inputs: the
// coefficients are formed in double so |O|^2 - r^2 keeps its low digits for large radii
// and grazing rays.  Only the two root values change; the disc sign test stays FP32 so the
// hit/miss topology matches the FP32 path unless the FP32 discriminant itself was wrong.
PHX_D void polish_roots(float& t1, float& t2, double d, double b, double c)
{
    double disc = b * b - d * c;
    if (disc <= 0.0) return;
    double sd = sqrt(disc);
    double q = b > 0.0 ? -(b + sd) : -(b - sd);
    double r1 = q / d, r2 = c / q;
    t1 = (float)fmin(r1, r2);
    t2 = (float)fmax(r1, r2);
}

// ---------------------------------------------------------------- leaves
template <bool POLISH>
PHX_D bool leaf_sphere(float4& isect, const float4& q0, float t_min, const float3& o, const float3& dir)
{
    float3 center = make_float3(q0.x, q0.y, q0.z);
    float radius = q0.w;
    float3 O = o - center;
    float3 D = dir;
    float b = dot(O, D);
    float c = dot(O, O) - radius * radius;
    float d = dot(D, D);
    float root1, root2, disc, sdisc;
    robust_roots(root1, root2, disc, sdisc, d, b, c);
    if (POLISH && sdisc > 0.f) {
        double ox = (double)o.x - center.x, oy = (double)o.y - center.y, oz = (double)o.z - center.z;
        double bb = ox * D.x + oy * D.y + oz * D.z;
        double cc = ox * ox + oy * oy + oz * oz - (double)radius * radius;
        double dd = (double)D.x * D.x + (double)D.y * D.y + (double)D.z * D.z;
        polish_roots(root1, root2, dd, bb, cc);
    }
    float t_cand = sdisc > 0.f ? (root1 > t_min ? root1 : root2) : t_min;
    bool valid = t_cand > t_min;
    if (valid) {
        isect.x = (O.x + t_cand * D.x) / radius;
        isect.y = (O.y + t_cand * D.y) / radius;
        isect.z = (O.z + t_cand * D.z) / radius;
        isect.w = t_cand;
    }
    return valid;
}

template <bool POLISH>
PHX_D bool leaf_zsphere(float4& isect, const float4& q0, const float4& q1, float t_min, const float3& o, const float3& dir)
{
    const float3 center = make_float3(q0.x, q0.y, q0.z);
    float3 O = o - center;
    float3 D = dir;
    const float radius = q0.w;
    float b = dot(O, D);
    float c = dot(O, O) - radius * radius;
    if (c > 0.f && b > 0.f) return false;   // outside and moving away
    const float zmax = center.z + q1.y;
    const float zmin = center.z + q1.x;
    float d = dot(D, D);
    float t1sph, t2sph, disc, sdisc;
    robust_roots(t1sph, t2sph, disc, sdisc, d, b, c);
    if (POLISH && sdisc > 0.f) {
        double ox = (double)o.x - center.x, oy = (double)o.y - center.y, oz = (double)o.z - center.z;
        double bb = ox * D.x + oy * D.y + oz * D.z;
        double cc = ox * ox + oy * oy + oz * oz - (double)radius * radius;
        double dd = (double)D.x * D.x + (double)D.y * D.y + (double)D.z * D.z;
        polish_roots(t1sph, t2sph, dd, bb, cc);
    }
    float z1sph = o.z + t1sph * dir.z;
    float z2sph = o.z + t2sph * dir.z;
    float idz = 1.f / dir.z;
    float t_QCAP = (zmax - o.z) * idz;
    float t_PCAP = (zmin - o.z) * idz;
    float t1cap = fminf(t_QCAP, t_PCAP);
    float t2cap = fmaxf(t_QCAP, t_PCAP);
    if (t1cap < t1sph || t1cap > t2sph) t1cap = t_min;
    if (t2cap < t1sph || t2cap > t2sph) t2cap = t_min;
    float t_cand = t_min;
    if (sdisc > 0.f) {
        if (t1sph > t_min && z1sph > zmin && z1sph <= zmax) t_cand = t1sph;
        else if (t1cap > t_min) t_cand = t1cap;
        else if (t2cap > t_min) t_cand = t2cap;
        else if (t2sph > t_min && z2sph > zmin && z2sph <= zmax) t_cand = t2sph;
    }
    bool valid = t_cand > t_min;
    if (valid) {
        isect.w = t_cand;
        if (t_cand == t1sph || t_cand == t2sph) {
            isect.x = (O.x + t_cand * D.x) / radius;
            isect.y = (O.y + t_cand * D.y) / radius;
            isect.z = (O.z + t_cand * D.z) / radius;
        } else {
            isect.x = 0.f;
            isect.y = 0.f;
            isect.z = t_cand == t_PCAP ? -1.f : 1.f;
        }
    }
    return valid;
}

template <bool POLISH>
PHX_D bool leaf_cylinder(float4& isect, const float4& q0, const float4& q1, float t_min, const float3& o, const float3& dir)
{
    const float r = q0.w;
    const float z1 = q1.x;
    const float z2 = q1.y;
    const float ox = o.x, oy = o.y, oz = o.z;
    const float vx = dir.x, vy = dir.y, vz = dir.z;
    const float r2 = r * r;
    const float a = vx * vx + vy * vy;
    const float b = ox * vx + oy * vy;
    const float c = ox * ox + oy * oy - r2;
    float t_near, t_far, disc, sdisc;
    robust_roots_disq(t_min, t_near, t_far, disc, sdisc, a, b, c);
    if (POLISH && sdisc > 0.f) {
        double aa = (double)vx * vx + (double)vy * vy;
        double bb = (double)ox * vx + (double)oy * vy;
        double cc = (double)ox * ox + (double)oy * oy - (double)r * r;
        polish_roots(t_near, t_far, aa, bb, cc);
    }
    float z_near = oz + t_near * vz;
    float z_far = oz + t_far * vz;
    const float t_z1cap = (z1 - oz) / vz;
    const float r2_z1cap = (ox + t_z1cap * vx) * (ox + t_z1cap * vx) + (oy + t_z1cap * vy) * (oy + t_z1cap * vy);
    const float t_z2cap = (z2 - oz) / vz;
    const float r2_z2cap = (ox + t_z2cap * vx) * (ox + t_z2cap * vx) + (oy + t_z2cap * vy) * (oy + t_z2cap * vy);
    const float INF = __int_as_float(0x7f800000);
    float t_cand = INF;
    if (t_near > t_min && z_near > z1 && z_near < z2 && t_near < t_cand) t_cand = t_near;
    if (t_far > t_min && z_far > z1 && z_far < z2 && t_far < t_cand) t_cand = t_far;
    if (t_z1cap > t_min && r2_z1cap <= r2 && t_z1cap < t_cand) t_cand = t_z1cap;
    if (t_z2cap > t_min && r2_z2cap <= r2 && t_z2cap < t_cand) t_cand = t_z2cap;
    bool valid = t_cand > t_min && t_cand < INF;
    if (valid) {
        bool sheet = (t_cand == t_near || t_cand == t_far);
        isect.x = sheet ? (ox + t_cand * vx) / r : 0.f;
        isect.y = sheet ? (oy + t_cand * vy) / r : 0.f;
        isect.z = sheet ? 0.f : (t_cand == t_z1cap ? -1.f : 1.f);
        isect.w = t_cand;
    }
    return valid;
}

PHX_COLD float4 leaf_box3(const float4 q0, const float t_min, const float3 o, const float3 dir)
{
    float4 isect = make_float4(0.f, 0.f, 0.f, 0.f);
    const float3 bmin = make_float3(-q0.x / 2.f, -q0.y / 2.f, -q0.z / 2.f);
    const float3 bmax = make_float3(q0.x / 2.f, q0.y / 2.f, q0.z / 2.f);
    float3 idir = f3s(1.f) / dir;
    float3 t0 = (bmin - o) * idir;
    float3 t1 = (bmax - o) * idir;
    float3 nr = fminf3(t0, t1);
    float3 fr = fmaxf3(t0, t1);
    float t_near = hmax(nr);
    float t_far = hmin(fr);
    bool along_x = dir.x != 0.f && dir.y == 0.f && dir.z == 0.f;
    bool along_y = dir.x == 0.f && dir.y != 0.f && dir.z == 0.f;
    bool along_z = dir.x == 0.f && dir.y == 0.f && dir.z != 0.f;
    bool in_x = o.x > bmin.x && o.x < bmax.x;
    bool in_y = o.y > bmin.y && o.y < bmax.y;
    bool in_z = o.z > bmin.z && o.z < bmax.z;
    bool has = false;
    if (along_x) has = in_y && in_z;
    else if (along_y) has = in_x && in_z;
    else if (along_z) has = in_x && in_y;
    else has = (t_far > t_near && t_far > 0.f);
    if (has) {
        float t_cand = t_min < t_near ? t_near : (t_min < t_far ? t_far : t_min);
        float3 p = o + t_cand * dir;
        float3 pa = make_float3(fabsf(p.x) / (bmax.x - bmin.x), fabsf(p.y) / (bmax.y - bmin.y), fabsf(p.z) / (bmax.z - bmin.z));
        float3 n = f3s(0.f);
        if (pa.x >= pa.y && pa.x >= pa.z) n.x = copysignf(1.f, p.x);
        else if (pa.y >= pa.x && pa.y >= pa.z) n.y = copysignf(1.f, p.y);
        else if (pa.z >= pa.x && pa.z >= pa.y) n.z = copysignf(1.f, p.z);
        if (t_cand > t_min) {   // valid: w > t_min
            isect.x = n.x; isect.y = n.y; isect.z = n.z; isect.w = t_cand;
        }
    }
    return isect;
}

// ---------------------------------------------------------------- torus (FP64)
// f(u) = (|p|^2 + R^2 - r^2)^2 - 4 R^2 (px^2 + py^2),  p = o + u*n  (|n| = 1)
// Real roots of the quartic are bracketed between the real roots of its derivative
// (a cubic, solved in closed form) and refined by safeguarded Newton/bisection.
PHX_D double q4eval(const double* c, double u) { return (((u + c[3]) * u + c[2]) * u + c[1]) * u + c[0]; }
PHX_D double q4deriv(const double* c, double u) { return ((4.0 * u + 3.0 * c[3]) * u + 2.0 * c[2]) * u + c[1]; }

// real roots of x^3 + a x^2 + b x + c, ascending; returns count
PHX_D int cubic_real_roots(double a, double b, double c, double* x)
{
    const double a3 = a / 3.0;
    const double p = b - a * a3;                       // depressed: t^3 + p t + q
    const double q = 2.0 * a3 * a3 * a3 - a3 * b + c;
    const double disc = 0.25 * q * q + p * p * p / 27.0;
    if (disc > 0.0) {
        double s = sqrt(disc);
        double A = cbrt(-0.5 * q + s);
        double B = cbrt(-0.5 * q - s);
        x[0] = A + B - a3;
        return 1;
    }
    if (p == 0.0) { x[0] = -a3; return 1; }
    double m = 2.0 * sqrt(-p / 3.0);
    double arg = 3.0 * q / (p * m);
    arg = fmin(1.0, fmax(-1.0, arg));
    double th = acos(arg) / 3.0;
    const double TWO_PI_3 = 2.0943951023931954923;
    double r0 = m * cos(th) - a3, r1 = m * cos(th - TWO_PI_3) - a3, r2 = m * cos(th - 2.0 * TWO_PI_3) - a3;
    // ascending
    if (r0 > r1) { double t = r0; r0 = r1; r1 = t; }
    if (r1 > r2) { double t = r1; r1 = r2; r2 = t; }
    if (r0 > r1) { double t = r0; r0 = r1; r1 = t; }
    x[0] = r0; x[1] = r1; x[2] = r2;
    return 3;
}

// smallest root of the monic quartic in (lo, hi]; returns false if none
PHX_D bool quartic_first_root(const double* c, double lo, double hi, double& root, unsigned& err)
{
    double crit[3];
    int nc = cubic_real_roots(0.75 * c[3], 0.5 * c[2], 0.25 * c[1], crit);
    double edges[5];
    int ne = 0;
    edges[ne++] = lo;
    for (int i = 0; i < nc; i++) if (crit[i] > lo && crit[i] < hi) edges[ne++] = crit[i];
    edges[ne++] = hi;
    for (int i = 0; i + 1 < ne; i++) {
        double a = edges[i], b = edges[i + 1];
        double fa = q4eval(c, a), fb = q4eval(c, b);
        if (fa == 0.0 && i > 0) { root = a; return true; }
        if ((fa < 0.0) == (fb < 0.0) && fb != 0.0) continue;
        // safeguarded Newton inside [a,b]
        double x = 0.5 * (a + b);
        int it = 0;
        for (; it < 100; it++) {
            double fx = q4eval(c, x);
            if (fx == 0.0) break;
            if ((fx < 0.0) == (fa < 0.0)) { a = x; fa = fx; } else { b = x; }
            double dfx = q4deriv(c, x);
            double xn = dfx != 0.0 ? x - fx / dfx : 0.5 * (a + b);
            if (!(xn > a && xn < b)) xn = 0.5 * (a + b);
            if (fabs(xn - x) <= 1e-12 * fmax(1.0, fabs(x))) { x = xn; break; }
            x = xn;
        }
        if (it == 100) err |= PHX_STATUS_LOOP_CAP;
        root = x;
        return true;
    }
    return false;
}

// q0.y = minor radius r (rmax), q0.z = major radius R (rtor) ; full phi range
PHX_COLD float4 leaf_torus(const float4 q0, const float t_min, const float3 o, const float3 dir)
{
    float4 isect = make_float4(0.f, 0.f, 0.f, 0.f);
    unsigned err = 0;
    const double r = q0.y, R = q0.z;
    const double dx = dir.x, dy = dir.y, dz = dir.z;
    const double dl = sqrt(dx * dx + dy * dy + dz * dz);
    if (!(dl > 0.0)) return isect;
    const double nx = dx / dl, ny = dy / dl, nz = dz / dl;
    double ox = o.x, oy = o.y, oz = o.z;
    // clip to the bounding sphere |p| <= R + r, and shift the origin near the torus
    const double Rb = R + r;
    const double bb = ox * nx + oy * ny + oz * nz;
    const double cc = ox * ox + oy * oy + oz * oz - Rb * Rb;
    const double dsc = bb * bb - cc;
    if (dsc <= 0.0) return isect;
    const double sq = sqrt(dsc);
    const double s_in = -bb - sq, s_out = -bb + sq;
    const double s_min = (double)t_min * dl;
    if (s_out <= s_min) return isect;
    const double s0 = fmax(s_in, 0.0);
    ox += s0 * nx; oy += s0 * ny; oz += s0 * nz;
    const double B = 2.0 * (ox * nx + oy * ny + oz * nz);
    const double C = ox * ox + oy * oy + oz * oz + R * R - r * r;
    const double R4 = 4.0 * R * R;
    double c[4];
    c[3] = 2.0 * B;
    c[2] = B * B + 2.0 * C - R4 * (nx * nx + ny * ny);
    c[1] = 2.0 * B * C - 2.0 * R4 * (ox * nx + oy * ny);
    c[0] = C * C - R4 * (ox * ox + oy * oy);
    const double lo = fmax(s_min - s0, 0.0);
    const double hi = s_out - s0 + 1e-9 * Rb;
    double u;
    if (!quartic_first_root(c, lo, hi, u, err)) return isect;
    const double s = s0 + u;
    const float t = (float)(s / dl);
    if (!(t > t_min)) return isect;
    const double px = ox + u * nx, py = oy + u * ny, pz = oz + u * nz;
    const double k = px * px + py * py + pz * pz + R * R - r * r;
    double gx = px * (k - 2.0 * R * R), gy = py * (k - 2.0 * R * R), gz = pz * k;
    const double gl = sqrt(gx * gx + gy * gy + gz * gz);
    isect.x = (float)(gx / gl);
    isect.y = (float)(gy / gl);
    isect.z = (float)(gz / gl);
    isect.w = t;
    return isect;
}

// ---------------------------------------------------------------- further leaves
// cone   CSG/csg_intersect_leaf_newcone.h        hyperboloid CSG/csg_intersect_leaf_hyperboloid.h
// convexpolyhedron CSG/csg_intersect_leaf_convexpolyhedron.h   phicut CSG/csg_intersect_leaf_phicut.h
// halfspace, slab, infcylinder, disc   CSG/csg_intersect_leaf_{halfspace,slab,infcylinder,disc}.h
// Each keeps the reference's order of FP32 operations (parity against its intersector).
#define PHX_RT_MAX 1.e27f

PHX_D float fmin4(float a, float b, float c, float d) { return fminf(fminf(a, b), fminf(c, d)); }

// cone frustum: q0 = (r1, z1, r2, z2), z2 > z1, with end caps
PHX_COLD float4 leaf_cone(const float4 q0, const float t_min, const float3 o, const float3 d)
{
    float4 isect = make_float4(0.f, 0.f, 0.f, 0.f);
    const float r1 = q0.x, z1 = q0.y, r2 = q0.z, z2 = q0.w;
    const float r1r1 = r1 * r1, r2r2 = r2 * r2;
    const float tth = (r2 - r1) / (z2 - z1);
    const float tth2 = tth * tth;
    const float z0 = (z2 * r1 - z1 * r2) / (r1 - r2);
    const float idz = 1.f / d.z;
    float t_cap1 = d.z == 0.f ? PHX_RT_MAX : (z1 - o.z) * idz;
    float t_cap2 = d.z == 0.f ? PHX_RT_MAX : (z2 - o.z) * idz;
    const float rr_cap1 = (o.x + t_cap1 * d.x) * (o.x + t_cap1 * d.x) + (o.y + t_cap1 * d.y) * (o.y + t_cap1 * d.y);
    const float rr_cap2 = (o.x + t_cap2 * d.x) * (o.x + t_cap2 * d.x) + (o.y + t_cap2 * d.y) * (o.y + t_cap2 * d.y);
    t_cap1 = rr_cap1 < r1r1 && t_cap1 > t_min ? t_cap1 : PHX_RT_MAX;
    t_cap2 = rr_cap2 < r2r2 && t_cap2 > t_min ? t_cap2 : PHX_RT_MAX;
    const float c2 = d.x * d.x + d.y * d.y - d.z * d.z * tth2;
    const float c1 = o.x * d.x + o.y * d.y - (o.z - z0) * d.z * tth2;
    const float c0 = o.x * o.x + o.y * o.y - (o.z - z0) * (o.z - z0) * tth2;
    float t_near, t_far, disc, sdisc;
    robust_roots_disq(PHX_RT_MAX, t_near, t_far, disc, sdisc, c2, c1, c0);
    const float z_near = o.z + t_near * d.z;
    const float z_far = o.z + t_far * d.z;
    t_near = z_near > z1 && z_near < z2 && t_near > t_min ? t_near : PHX_RT_MAX;
    t_far = z_far > z1 && z_far < z2 && t_far > t_min ? t_far : PHX_RT_MAX;
    const float t_cand = fmin4(t_near, t_far, t_cap1, t_cap2);
    if (t_cand > t_min && t_cand < PHX_RT_MAX) {
        if (t_cand == t_cap1 || t_cand == t_cap2) {
            isect.z = t_cand == t_cap2 ? 1.f : -1.f;
        } else {
            const float3 n = normalize(make_float3(o.x + t_cand * d.x, o.y + t_cand * d.y, (z0 - (o.z + t_cand * d.z)) * tth2));
            isect.x = n.x; isect.y = n.y; isect.z = n.z;
        }
        isect.w = t_cand;
    }
    return isect;
}

// one-sheet hyperboloid x^2 + y^2 = r0^2 ((z/zf)^2 + 1) between z1 < z2: q0 = (r0, zf, z1, z2)
PHX_COLD float4 leaf_hyperboloid(const float4 q0, const float t_min, const float3 o, const float3 s)
{
    float4 isect = make_float4(0.f, 0.f, 0.f, 0.f);
    const float r0 = q0.x, zf = q0.y, z1 = q0.z, z2 = q0.w;
    const float rr0 = r0 * r0;
    const float z1s = z1 / zf, z2s = z2 / zf;
    const float rr1 = rr0 * (z1s * z1s + 1.f);
    const float rr2 = rr0 * (z2s * z2s + 1.f);
    const float A = -rr0 / (zf * zf);
    const float B = -rr0;
    const float dd = s.x * s.x + s.y * s.y + A * s.z * s.z;
    const float b = o.x * s.x + o.y * s.y + A * o.z * s.z;
    const float c = o.x * o.x + o.y * o.y + A * o.z * o.z + B;
    float t1hyp, t2hyp, disc, sdisc;
    robust_roots(t1hyp, t2hyp, disc, sdisc, dd, b, c);
    const float h1z = o.z + t1hyp * s.z;
    const float h2z = o.z + t2hyp * s.z;
    const float osz = 1.f / s.z;
    const float t2cap = (z2 - o.z) * osz;
    const float t1cap = (z1 - o.z) * osz;
    const float3 c1 = o + t1cap * s;
    const float3 c2 = o + t2cap * s;
    const float crr1 = c1.x * c1.x + c1.y * c1.y;
    const float crr2 = c2.x * c2.x + c2.y * c2.y;
    const float a0 = t1hyp > t_min && disc > 0.f && h1z > z1 && h1z < z2 ? t1hyp : PHX_RT_MAX;
    const float a1 = t2hyp > t_min && disc > 0.f && h2z > z1 && h2z < z2 ? t2hyp : PHX_RT_MAX;
    const float a2 = t2cap > t_min && crr2 < rr2 ? t2cap : PHX_RT_MAX;
    const float a3 = t1cap > t_min && crr1 < rr1 ? t1cap : PHX_RT_MAX;
    const float t_cand = fmin4(a0, a1, a2, a3);
    if (t_cand > t_min && t_cand < PHX_RT_MAX) {
        isect.w = t_cand;
        if (t_cand == t1hyp || t_cand == t2hyp) {
            const float3 p = o + t_cand * s;
            const float3 n = normalize(make_float3(p.x, p.y, A * p.z));
            isect.x = n.x; isect.y = n.y; isect.z = n.z;
        } else {
            isect.z = t_cand == t1cap ? -1.f : 1.f;
        }
    }
    return isect;
}

// convex polyhedron: the intersection of planeNum half-spaces n.x <= w from the plan table, starting
// at planeIdx (q0 words x, y); entering keeps the latest entry, exiting the earliest exit
PHX_COLD float4 leaf_convexpolyhedron(const float4 q0, const float4* __restrict__ plan, const float t_min, const float3 o, const float3 d)
{
    float4 isect = make_float4(0.f, 0.f, 0.f, 0.f);
    const unsigned planeIdx = __float_as_uint(q0.x), planeNum = __float_as_uint(q0.y);
    const float INF = __int_as_float(0x7f800000);
    float t0 = -INF, t1 = INF;
    float3 n0 = make_float3(0.f, 0.f, 0.f), n1 = make_float3(0.f, 0.f, 0.f);
    for (unsigned i = 0; i < planeNum; i++) {       // planeIdx + planeNum <= num_plan, checked at phx_create
        const float4 pl = __ldg(plan + planeIdx + i);
        const float3 n = make_float3(pl.x, pl.y, pl.z);
        const float nd = dot(n, d);
        const float no = dot(n, o);
        const float dist = no - pl.w;
        const float t_cand = -dist / nd;
        if (nd == 0.f && dist < 0.f) continue;          // parallel, inside this half-space
        if (nd == 0.f && dist > 0.f) return isect;      // parallel, outside: no intersect
        if (nd < 0.f) { if (t_cand > t0) { t0 = t_cand; n0 = n; } }
        else          { if (t_cand < t1) { t1 = t_cand; n1 = n; } }
    }
    if (t0 < t1) {
        if (t0 > t_min) isect = make_float4(n0.x, n0.y, n0.z, t0);
        else if (t1 > t_min) isect = make_float4(n1.x, n1.y, n1.z, t1);
        else isect.w = -0.f;     // the reference reports this valid with isect unset: w = -0 carries that
    }
    return isect;
}

// a leaf's validity as the reference reports it: t > t_min, or the convexpolyhedron's valid
// report with isect unset (w = -0).  Only the DISCONTIGUOUS list reads validity without t.
PHX_D bool phx_leaf_valid(const float4& is, float t_min) { return is.w > t_min || __float_as_uint(is.w) == 0x80000000u; }

// phi wedge between the half-planes at phi0 and phi1: q0 = (cos phi0, sin phi0, cos phi1, sin phi1);
// a miss with an unbounded exit carries y = -0 (promoted to EXIT by the tree evaluator)
PHX_COLD float4 leaf_phicut(const float4 q0, const float t_min, const float3 o, const float3 d)
{
    float4 isect = make_float4(0.f, 0.f, 0.f, 0.f);
    const float cosPhi0 = q0.x, sinPhi0 = q0.y, cosPhi1 = q0.z, sinPhi1 = q0.w;
    const float d_n0 = d.x * sinPhi0 + d.y * (-cosPhi0);
    const float d_n1 = d.x * (-sinPhi1) + d.y * (cosPhi1);
    const float o_n0 = o.x * sinPhi0 + o.y * (-cosPhi0);
    const float o_n1 = o.x * (-sinPhi1) + o.y * (cosPhi1);
    float t0 = d_n0 == 0.f ? t_min : -o_n0 / d_n0;
    float t1 = d_n1 == 0.f ? t_min : -o_n1 / d_n1;
    const float PR = d_n0 == 0.f ? -o_n0 : -d_n0;
    const float QR = d_n1 == 0.f ? -o_n1 : -d_n1;
    const float PQ = cosPhi0 * sinPhi1 - cosPhi1 * sinPhi0;
    const bool unbounded_exit = PQ >= 0.f ? (PR >= 0.f && QR <= 0.f) : (PR >= 0.f || QR <= 0.f);
    const float side0 = o.x * cosPhi0 + o.y * sinPhi0 + (d.x * cosPhi0 + d.y * sinPhi0) * t0;
    const float side1 = o.x * cosPhi1 + o.y * sinPhi1 + (d.x * cosPhi1 + d.y * sinPhi1) * t1;
    if (side0 < 0.f) t0 = t_min;
    if (side1 < 0.f) t1 = t_min;
    const float t_near = fminf(t0, t1);
    const float t_far = fmaxf(t0, t1);
    const float t_cand = t_near > t_min ? t_near : (t_far > t_min ? t_far : t_min);
    if (t_cand > t_min) {
        isect.x = t_cand == t1 ? -sinPhi1 : sinPhi0;
        isect.y = t_cand == t1 ? cosPhi1 : -cosPhi0;
        isect.w = t_cand;
    } else if (unbounded_exit) {
        isect.y = -isect.y;
    }
    return isect;
}

// half-space n.x <= w: q0 = (n, w); a miss from inside carries y = -0 (unbounded exit)
PHX_COLD float4 leaf_halfspace(const float4 q0, const float t_min, const float3 o, const float3 d)
{
    float4 isect = make_float4(0.f, 0.f, 0.f, 0.f);
    const float3 n = make_float3(q0.x, q0.y, q0.z);
    const float on = dot(o, n);
    const float dn = dot(d, n);
    const float on_w = on - q0.w;
    const bool inside = on_w < -1e-9f;
    const float t = fabsf(dn) > 0.f ? -on_w / dn : t_min;
    if (t > t_min) isect = make_float4(n.x, n.y, n.z, t);
    else if (inside) isect.y = -0.f;
    return isect;
}

// slab a <= n.x <= b: q0 = n, q1 = (a, b)
PHX_COLD float4 leaf_slab(const float4 q0, const float4 q1, const float t_min, const float3 o, const float3 d)
{
    float4 isect = make_float4(0.f, 0.f, 0.f, 0.f);
    const float3 n = make_float3(q0.x, q0.y, q0.z);
    const float idn = 1.f / dot(d, n);
    const float on = dot(o, n);
    const float ta = (q1.x - on) * idn;
    const float tb = (q1.y - on) * idn;
    const float t_near = fminf(ta, tb);
    const float t_far = fmaxf(ta, tb);
    const float t_cand = t_near > t_min ? t_near : (t_far > t_min ? t_far : t_min);
    if (t_cand > t_min) {
        const bool b_hit = t_cand == tb;
        isect = make_float4(b_hit ? n.x : -n.x, b_hit ? n.y : -n.y, b_hit ? n.z : -n.z, t_cand);
    }
    return isect;
}

// infinite cylinder about z of radius q0.w
PHX_COLD float4 leaf_infcylinder(const float4 q0, const float t_min, const float3 O, const float3 D)
{
    float4 isect = make_float4(0.f, 0.f, 0.f, 0.f);
    const float r = q0.w;
    const float a = D.x * D.x + D.y * D.y;
    const float b = O.x * D.x + O.y * D.y;
    const float c = O.x * O.x + O.y * O.y - r * r;
    const float disc0 = b * b - a * c;
    if (disc0 > 0.f) {
        float t_NEAR, t_FAR, disc, sdisc;
        robust_roots(t_NEAR, t_FAR, disc, sdisc, a, b, c);
        const float t_cand = sdisc > 0.f ? (t_NEAR > t_min ? t_NEAR : t_FAR) : t_min;
        if (t_cand > t_min) isect = make_float4((O.x + t_cand * D.x) / r, (O.y + t_cand * D.y) / r, 0.f, t_cand);
    }
    return isect;
}

// annular disc of thickness z2 - z1 about (q0.x, q0.y, (z1+z2)/2), inner radius q0.z, outer q0.w
PHX_COLD float4 leaf_disc(const float4 q0, const float4 q1, const float t_min, const float3 ray_origin, const float3 n)
{
    float4 isect = make_float4(0.f, 0.f, 0.f, 0.f);
    const float inner = q0.z, radius = q0.w, z1 = q1.x, z2 = q1.y;
    const float zc = (z1 + z2) / 2.f;
    const float zdelta = (z2 - z1) / 2.f;
    const float3 center = make_float3(q0.x, q0.y, zc);
    const float3 m = ray_origin - center;
    const float3 dn = make_float3(0.f, 0.f, 1.f);
    const float rr = radius * radius, ii = inner * inner;
    const float mm = dot(m, m), nn = dot(n, n), nd = dot(n, dn), md = dot(m, dn), mn = dot(m, n);
    const float t_center = -md / nd;
    const float rsq = t_center * (2.f * mn + t_center * nn) + mm;
    const float t_delta = nd < 0.f ? -zdelta / nd : zdelta / nd;
    const float root1 = t_center - t_delta;
    const float root2 = t_center + t_delta;
    const float t_cand = (rsq < rr && rsq > ii) ? (root1 > t_min ? root1 : root2) : t_min;
    const float side = md + t_cand * nd;
    if (t_cand > t_min) isect = make_float4(0.f, 0.f, side > 0.f ? 1.f : -1.f, t_cand);
    return isect;
}

// ---------------------------------------------------------------- leaf with transform
#if PHX_OUTLINE
#define PHX_LEAFFN __device__ __noinline__
#else
#define PHX_LEAFFN __device__ __forceinline__
#endif
// One out-of-line copy of the leaf intersector, shared by the tree evaluator and leaf-rooted
// prims; arguments and result by value so nothing goes through the stack.  A miss returns w=0
// (with x=-0 for a complemented leaf), a hit has w = t > t_min.
// transform of the ray into the leaf frame and of the normal back, and the complement, around
// one leaf intersector (CSG/csg_intersect_leaf.h:174-300)
#define PHX_LEAF_PROLOGUE                                                                        \
    float4 isect = make_float4(0.f, 0.f, 0.f, 0.f);                                              \
    const float4 q0 = __ldg(node + 4 * ni + 0);                                                  \
    const float4 q1 = __ldg(node + 4 * ni + 1);                                                  \
    const float4 q3 = __ldg(node + 4 * ni + 3);                                                  \
    const unsigned typecode = __float_as_uint(q3.z);                                             \
    const unsigned tc_w = __float_as_uint(q3.w);                                                 \
    const unsigned gtransformIdx = tc_w & 0x7fffffffu;                                           \
    const bool complement = (tc_w & 0x80000000u) != 0u;                                          \
    float4 t4[4];                                                                                \
    const float4* q = nullptr;                                                                   \
    if (gtransformIdx > 0) {                                                                     \
        const float4* src = itra + 4 * (gtransformIdx - 1);                                      \
        t4[0] = __ldg(src + 0); t4[1] = __ldg(src + 1); t4[2] = __ldg(src + 2); t4[3] = __ldg(src + 3); \
        q = t4;                                                                                  \
    }                                                                                            \
    float3 origin = q ? xform_row(q, ray_o, 1.f) : ray_o;                                        \
    float3 direction = q ? xform_row(q, ray_d, 0.f) : ray_d;                                     \
    bool valid = false;

#define PHX_LEAF_EPILOGUE                                                                        \
    if (valid && q) {                                                                            \
        float3 n = xform_col(q, make_float3(isect.x, isect.y, isect.z), 0.f);                    \
        isect.x = n.x; isect.y = n.y; isect.z = n.z;                                             \
    }                                                                                            \
    if (complement) {                                                                            \
        isect.x = valid ? -isect.x : -0.f;                                                       \
        isect.y = valid ? -isect.y : isect.y;                                                    \
        isect.z = valid ? -isect.z : isect.z;                                                    \
    }                                                                                            \
    return isect;

// the five base leaves
template <bool POLISH>
PHX_LEAFFN float4 leaf_eval(const float4* __restrict__ node, const float4* __restrict__ itra, const int ni, const float t_min,
                            const float3 ray_o, const float3 ray_d)
{
    PHX_LEAF_PROLOGUE
    switch (typecode) {
        case PHX_CSG_SPHERE:   valid = leaf_sphere<POLISH>(isect, q0, t_min, origin, direction); break;
        case PHX_CSG_ZSPHERE:  valid = leaf_zsphere<POLISH>(isect, q0, q1, t_min, origin, direction); break;
        case PHX_CSG_CYLINDER: valid = leaf_cylinder<POLISH>(isect, q0, q1, t_min, origin, direction); break;
        case PHX_CSG_BOX3:     isect = leaf_box3(q0, t_min, origin, direction); valid = isect.w > t_min; break;
        case PHX_CSG_TORUS:    isect = leaf_torus(q0, t_min, origin, direction); valid = isect.w > t_min; break;
        default: break;
    }
    PHX_LEAF_EPILOGUE
}

// every leaf (the full variant)
template <bool POLISH>
PHX_LEAFFN float4 leaf_eval_full(const float4* __restrict__ node, const float4* __restrict__ itra, const float4* __restrict__ plan,
                                 const int ni, const float t_min, const float3 ray_o, const float3 ray_d)
{
    PHX_LEAF_PROLOGUE
    switch (typecode) {
        case PHX_CSG_SPHERE:   valid = leaf_sphere<POLISH>(isect, q0, t_min, origin, direction); break;
        case PHX_CSG_ZSPHERE:  valid = leaf_zsphere<POLISH>(isect, q0, q1, t_min, origin, direction); break;
        case PHX_CSG_CYLINDER: valid = leaf_cylinder<POLISH>(isect, q0, q1, t_min, origin, direction); break;
        case PHX_CSG_BOX3:     isect = leaf_box3(q0, t_min, origin, direction); valid = isect.w > t_min; break;
        case PHX_CSG_TORUS:    isect = leaf_torus(q0, t_min, origin, direction); valid = isect.w > t_min; break;
        case PHX_CSG_CONE:     isect = leaf_cone(q0, t_min, origin, direction); valid = isect.w > t_min; break;
        case PHX_CSG_HYPERBOLOID: isect = leaf_hyperboloid(q0, t_min, origin, direction); valid = isect.w > t_min; break;
        case PHX_CSG_CONVEXPOLYHEDRON: isect = leaf_convexpolyhedron(q0, plan, t_min, origin, direction); valid = isect.w > t_min; break;
        case PHX_CSG_PHICUT:   isect = leaf_phicut(q0, t_min, origin, direction); valid = isect.w > t_min; break;
        case PHX_CSG_HALFSPACE: isect = leaf_halfspace(q0, t_min, origin, direction); valid = isect.w > t_min; break;
        case PHX_CSG_SLAB:     isect = leaf_slab(q0, q1, t_min, origin, direction); valid = isect.w > t_min; break;
        case PHX_CSG_INFCYLINDER: isect = leaf_infcylinder(q0, t_min, origin, direction); valid = isect.w > t_min; break;
        case PHX_CSG_DISC:     isect = leaf_disc(q0, q1, t_min, origin, direction); valid = isect.w > t_min; break;
        default: break;
    }
    // w = -0: the convexpolyhedron's valid report with isect unset, kept valid as the reference does
    valid = valid || __float_as_uint(isect.w) == 0x80000000u;
    PHX_LEAF_EPILOGUE
}

// one leaf through the evaluator of the variant
template <int CV>
PHX_D float4 leaf_call(const PhxCsgCtx& g, int ni, float t_min, const float3& o, const float3& d)
{
    if constexpr (PHX_CV_F(CV)) return leaf_eval_full<PHX_CV_P(CV)>(g.node, g.itra, g.plan, ni, t_min, o, d);
    else return leaf_eval<PHX_CV_P(CV)>(g.node, g.itra, ni, t_min, o, d);
}

template <int CV>
PHX_D bool intersect_leaf(float4& isect, const PhxCsgCtx& g, int ni, float t_min, const float3& ray_o, const float3& ray_d, unsigned& err)
{
    (void)err;
    isect = leaf_call<CV>(g, ni, t_min, ray_o, ray_d);
    return isect.w > t_min;
}

PHX_D int phx_classify(const float4& ise, const float3& d, float tmin)
{
    return fabsf(ise.w) > tmin ? (ise.x * d.x + ise.y * d.y + ise.z * d.z < 0.f ? PHX_STATE_ENTER : PHX_STATE_EXIT) : PHX_STATE_MISS;
}

// ---------------------------------------------------------------- list nodes
// CSG/csg_intersect_node.h:392-945.  A list header (typecode CONTIGUOUS, DISCONTIGUOUS or
// OVERLAP; q0.u.x = subNum, q0.u.y = subOffset) names subNum leaves at root + subOffset + i,
// root being the prim's first node (a list is a prim root, or a leaf of a boolean tree whose
// sub-nodes follow the complete binary tree).  Ranges are checked at phx_create.
#define PHX_LIST_MAX_ENTER 8

// union of leaves that may touch or overlap: the farthest exit reachable through a chain of
// overlapping constituents (CSG/csg_intersect_node.h:392-600)
template <int CV>
PHX_D bool intersect_list_contiguous(float4& isect, const PhxCsgCtx& g, int first, int num_sub, float t_min, const float3& o,
                                     const float3& d, unsigned& err)
{
    float4 nearest_enter = make_float4(0.f, 0.f, 0.f, PHX_RT_MAX);
    float4 farthest_exit = make_float4(0.f, 0.f, 0.f, t_min);
    int exit_count = 0;
    for (int i = 0; i < num_sub; i++) {
        const float4 s = leaf_call<CV>(g, first + i, t_min, o, d);
        if (!phx_leaf_valid(s, t_min)) continue;
        const int st = phx_classify(s, d, t_min);
        if (st == PHX_STATE_ENTER) { if (s.w < nearest_enter.w) nearest_enter = s; }
        else if (st == PHX_STATE_EXIT) exit_count += 1;
    }
    if (exit_count == 0) {
        const bool valid = nearest_enter.w > t_min && nearest_enter.w < PHX_RT_MAX;
        if (valid) isect = nearest_enter;
        return valid;
    }
    int enter_count = 0;
    float enter[PHX_LIST_MAX_ENTER];
    int aux[PHX_LIST_MAX_ENTER];
    for (int i = 0; i < num_sub; i++) {
        const float4 s = leaf_call<CV>(g, first + i, t_min, o, d);
        if (!phx_leaf_valid(s, t_min)) continue;
        const int st = phx_classify(s, d, t_min);
        if (st == PHX_STATE_ENTER) {
            // the reference's arrays hold 8 enters; more is undefined there: flag and drop
            if (enter_count >= PHX_LIST_MAX_ENTER) { err |= PHX_STATUS_CSG_STACK; continue; }
            aux[enter_count] = i;
            enter[enter_count] = s.w;
            enter_count += 1;
        } else if (st == PHX_STATE_EXIT) {
            exit_count += 1;
            if (s.w > farthest_exit.w) farthest_exit = s;
        }
    }
    // stable insertion sort of the enters by distance
    for (int i = 1; i < enter_count; i++) {
        const float ke = enter[i];
        const int ka = aux[i];
        int j = i - 1;
        while (j >= 0 && enter[j] > ke) { enter[j + 1] = enter[j]; aux[j + 1] = aux[j]; j--; }
        enter[j + 1] = ke;
        aux[j + 1] = ka;
    }
    for (int i = 0; i < enter_count; i++) {
        const float tminAdvanced = enter[i] + PHX_CSG_PROPAGATE_EPSILON;
        if (tminAdvanced < farthest_exit.w) {
            const float4 s = leaf_call<CV>(g, first + aux[i], tminAdvanced, o, d);
            if (phx_leaf_valid(s, tminAdvanced) && phx_classify(s, d, tminAdvanced) == PHX_STATE_EXIT) {
                exit_count += 1;
                if (s.w > farthest_exit.w) farthest_exit = s;
            }
        }
    }
    const bool valid = exit_count > 0 && farthest_exit.w > t_min;
    if (valid) isect = farthest_exit;
    return valid;
}

// union of disjoint leaves: the closest valid report (CSG/csg_intersect_node.h:654-700)
template <int CV>
PHX_D bool intersect_list_discontiguous(float4& isect, const PhxCsgCtx& g, int first, int num_sub, float t_min, const float3& o,
                                        const float3& d)
{
    float4 closest = make_float4(0.f, 0.f, 0.f, PHX_RT_MAX);
    for (int i = 0; i < num_sub; i++) {
        const float4 s = leaf_call<CV>(g, first + i, t_min, o, d);
        if (phx_leaf_valid(s, t_min) && s.w < closest.w) closest = s;
    }
    const bool valid = closest.w < PHX_RT_MAX;
    if (valid) isect = closest;
    return valid;
}

// intersection of leaves: farthest enter or nearest exit when every leaf is entered or exited
// and the farthest enter precedes the nearest exit (CSG/csg_intersect_node.h:819-910)
template <int CV>
PHX_D bool intersect_list_overlap(float4& isect, const PhxCsgCtx& g, int first, int num_sub, float t_min, const float3& o,
                                  const float3& d)
{
    float4 farthest_enter = make_float4(0.f, 0.f, 0.f, t_min);
    float4 nearest_exit = make_float4(0.f, 0.f, 0.f, PHX_RT_MAX);
    int enter_count = 0, exit_count = 0;
    for (int i = 0; i < num_sub; i++) {
        float4 s = leaf_call<CV>(g, first + i, t_min, o, d);
        if (!phx_leaf_valid(s, t_min)) continue;
        const int st = phx_classify(s, d, t_min);
        if (st == PHX_STATE_ENTER) {
            enter_count += 1;
            if (s.w > farthest_enter.w) farthest_enter = s;
            const float tminAdvanced = s.w + PHX_CSG_PROPAGATE_EPSILON;
            s = leaf_call<CV>(g, first + i, tminAdvanced, o, d);
            if (phx_leaf_valid(s, tminAdvanced) && phx_classify(s, d, tminAdvanced) == PHX_STATE_EXIT) {
                exit_count += 1;
                if (s.w < nearest_exit.w) nearest_exit = s;
            }
        } else if (st == PHX_STATE_EXIT) {
            exit_count += 1;
            if (s.w < nearest_exit.w) nearest_exit = s;
        }
    }
    const bool overlap_all = farthest_enter.w < nearest_exit.w && max(enter_count, exit_count) == num_sub;
    if (overlap_all) {
        if (farthest_enter.w > t_min && farthest_enter.w < PHX_RT_MAX) { isect = farthest_enter; return true; }
        if (nearest_exit.w > t_min && nearest_exit.w < PHX_RT_MAX) { isect = nearest_exit; return true; }
    }
    return false;
}

// list header ni, sub-nodes relative to the prim root; isect is untouched on a miss
template <int CV>
PHX_D bool intersect_list(float4& isect, const PhxCsgCtx& g, int ni, int root, unsigned typecode, float t_min, const float3& o,
                          const float3& d, unsigned& err)
{
    const float4 q0 = __ldg(g.node + 4 * ni);
    const int num_sub = (int)__float_as_uint(q0.x);
    const int first = root + (int)__float_as_uint(q0.y);
    switch (typecode) {
        case PHX_CSG_CONTIGUOUS: return intersect_list_contiguous<CV>(isect, g, first, num_sub, t_min, o, d, err);
        case PHX_CSG_DISCONTIGUOUS: return intersect_list_discontiguous<CV>(isect, g, first, num_sub, t_min, o, d);
        case PHX_CSG_OVERLAP: return intersect_list_overlap<CV>(isect, g, first, num_sub, t_min, o, d);
        default: return false;
    }
}

#define PHX_POSTORDER_NEXT(i, elev) (((i) & 1u) ? (i) >> 1 : ((i) << (elev)) + (1u << (elev)))

// ---------------------------------------------------------------- one-operator tree
// The postorder walk below specialised to a 3-node tree (operator over two leaves, e.g. a PMT
// cap U neck) with both intermediate results in registers.  It takes the same steps as the
// general evaluator: both leaves at t_min, combine at t_min; LOOP_A/LOOP_B re-intersect only
// the looping leaf from |t|+0.0001 (the left tranche (2,3) / right tranche (3,1) of
// CSG/csg_intersect_tree.h) and combine again at t_min.
#ifndef PHX_TREE3
#define PHX_TREE3 1
#endif
#define PHX_TREE3_LOOP_CAP 64

template <int CV>
PHX_D bool intersect_tree3(float4& isect, const PhxCsgCtx& g, int root, unsigned op, float t_min, const float3& o, const float3& d, unsigned& err)
{
    float4 L = leaf_call<CV>(g, root + 1, t_min, o, d);
    float4 R = leaf_call<CV>(g, root + 2, t_min, o, d);
    for (int it = 0; it < PHX_TREE3_LOOP_CAP; it++) {
        int l_state = phx_classify(L, d, t_min);
        int r_state = phx_classify(R, d, t_min);
        bool leftIsCloser = fabsf(L.w) <= fabsf(R.w);
        const bool l_promote = l_state == PHX_STATE_MISS && (signbit(L.x) || signbit(L.y));
        const bool r_promote = r_state == PHX_STATE_MISS && (signbit(R.x) || signbit(R.y));
        if (r_promote) { r_state = PHX_STATE_EXIT; leftIsCloser = true; }
        if (l_promote) { l_state = PHX_STATE_EXIT; leftIsCloser = false; }
        const int ctrl = phx_csg_lookup((int)op, l_state, r_state, leftIsCloser);
        if (ctrl < PHX_CTRL_LOOP_A) {
            float4 result = ctrl == PHX_CTRL_RETURN_MISS ? make_float4(0.f, 0.f, 0.f, 0.f) : (ctrl == PHX_CTRL_RETURN_A ? L : R);
            if (ctrl == PHX_CTRL_RETURN_FLIP_B) { result.x = -result.x; result.y = -result.y; result.z = -result.z; }
            result.w = copysignf(result.w, 1.f);
            isect = result;
            return isect.w > 0.f;
        }
        if (ctrl == PHX_CTRL_LOOP_A) L = leaf_call<CV>(g, root + 1, fabsf(L.w) + PHX_CSG_PROPAGATE_EPSILON, o, d);
        else R = leaf_call<CV>(g, root + 2, fabsf(R.w) + PHX_CSG_PROPAGATE_EPSILON, o, d);
    }
    err |= PHX_STATUS_CSG_STACK;
    isect = make_float4(0.f, 0.f, 0.f, 0.f);
    return false;
}

// ---------------------------------------------------------------- tree
template <int CV>
PHX_D bool intersect_tree(float4& isect, const PhxCsgCtx& g, int root, float t_min, const float3& o, const float3& d, unsigned& err)
{
    const unsigned numNode = __float_as_uint(__ldg(g.node + 4 * root).x);   // subNum
#if PHX_TREE3
    if (numNode == 3u) {
        const unsigned op = __float_as_uint(__ldg(g.node + 4 * root + 3).z);
        const unsigned tl = __float_as_uint(__ldg(g.node + 4 * (root + 1) + 3).z);
        const unsigned tr = __float_as_uint(__ldg(g.node + 4 * (root + 2) + 3).z);
        if (op >= PHX_CSG_UNION && op <= PHX_CSG_DIFFERENCE && tl >= PHX_CSG_LEAF && tr >= PHX_CSG_LEAF)
            return intersect_tree3<CV>(isect, g, root, op, t_min, o, d, err);
    }
#endif
    const unsigned height = (unsigned)(__ffs((int)numNode + 1) - 2);
    float4 stk[PHX_CSG_STACK];
    int sp = -1;
    unsigned tslice[PHX_TRANCHE_STACK];
    float ttmin[PHX_TRANCHE_STACK];
    int tp = 0;
    tslice[0] = ((1u << height) << 16) | 0u;
    ttmin[0] = t_min;
    unsigned ierr = 0;
    while (tp > -1) {
        const unsigned slice = tslice[tp];
        const float tmin = ttmin[tp];
        tp--;
        const unsigned beginIdx = slice >> 16;
        const unsigned endIdx = slice & 0xffffu;
        unsigned nodeIdx = beginIdx;
        while (nodeIdx != endIdx) {
            const unsigned depth = 31u - __clz(nodeIdx);
            const unsigned elevation = height - depth;
            const int ni = root + (int)nodeIdx - 1;
            const unsigned typecode = __float_as_uint(__ldg(g.node + 4 * ni + 3).z);
            if (typecode == PHX_CSG_ZERO) { nodeIdx = PHX_POSTORDER_NEXT(nodeIdx, elevation); continue; }
            if (typecode >= PHX_CSG_NODE) {
                float4 nd_isect = make_float4(0.f, 0.f, 0.f, 0.f);
                if constexpr (PHX_CV_F(CV)) {
                    if (typecode < PHX_CSG_LEAF) intersect_list<CV>(nd_isect, g, ni, root, typecode, tmin, o, d, err);
                    else intersect_leaf<CV>(nd_isect, g, ni, tmin, o, d, err);
                } else {
                    intersect_leaf<CV>(nd_isect, g, ni, tmin, o, d, err);   // lists launch the full variant
                }
                nd_isect.w = copysignf(nd_isect.w, nodeIdx % 2u == 0u ? -1.f : 1.f);
                if (sp >= PHX_CSG_STACK - 1) { ierr |= PHX_CSG_ERR_OVERFLOW; break; }
                stk[++sp] = nd_isect;
            } else {
                if (sp < 1) { ierr |= PHX_CSG_ERR_POP_EMPTY; break; }
                const bool firstLeft = signbit(stk[sp].w);
                const bool secondLeft = signbit(stk[sp - 1].w);
                if (!(firstLeft ^ secondLeft)) { ierr |= PHX_CSG_ERR_XOR_SIDE; break; }
                const int left = firstLeft ? sp : sp - 1;
                const int right = firstLeft ? sp - 1 : sp;
                const float4 L = stk[left];
                const float4 Rr = stk[right];
                int l_state = phx_classify(L, d, tmin);
                int r_state = phx_classify(Rr, d, tmin);
                const float t_left = fabsf(L.w);
                const float t_right = fabsf(Rr.w);
                bool leftIsCloser = t_left <= t_right;
                const bool l_promote = l_state == PHX_STATE_MISS && (signbit(L.x) || signbit(L.y));
                const bool r_promote = r_state == PHX_STATE_MISS && (signbit(Rr.x) || signbit(Rr.y));
                if (r_promote) { r_state = PHX_STATE_EXIT; leftIsCloser = true; }
                if (l_promote) { l_state = PHX_STATE_EXIT; leftIsCloser = false; }
                const int ctrl = phx_csg_lookup((int)typecode, l_state, r_state, leftIsCloser);
                if (ctrl < PHX_CTRL_LOOP_A) {
                    float4 result = ctrl == PHX_CTRL_RETURN_MISS ? make_float4(0.f, 0.f, 0.f, 0.f) : (ctrl == PHX_CTRL_RETURN_A ? L : Rr);
                    if (ctrl == PHX_CTRL_RETURN_FLIP_B) { result.x = -result.x; result.y = -result.y; result.z = -result.z; }
                    result.w = copysignf(result.w, nodeIdx % 2u == 0u ? -1.f : 1.f);
                    sp -= 2;
                    stk[++sp] = result;
                } else {
                    const bool loopA = ctrl == PHX_CTRL_LOOP_A;
                    const float4 loopv = loopA ? L : Rr;
                    const float4 other = loopA ? Rr : L;
                    const unsigned leftIdx = 2u * nodeIdx;
                    const unsigned rightIdx = leftIdx + 1u;
                    const unsigned otherIdx = loopA ? rightIdx : leftIdx;
                    (void)otherIdx;
                    const float tminAdvanced = fabsf(loopv.w) + PHX_CSG_PROPAGATE_EPSILON;
                    sp -= 2;
                    stk[++sp] = other;
                    const unsigned endTree = (nodeIdx << 16) | endIdx;
                    const unsigned leftTree = ((leftIdx << (elevation - 1u)) << 16) | (rightIdx << (elevation - 1u));
                    const unsigned rightTree = ((rightIdx << (elevation - 1u)) << 16) | nodeIdx;
                    const unsigned loopTree = loopA ? leftTree : rightTree;
                    if (tp >= PHX_TRANCHE_STACK - 1) { ierr |= PHX_CSG_ERR_TRANCHE; break; }
                    tp++; tslice[tp] = endTree; ttmin[tp] = tmin;
                    if (tp >= PHX_TRANCHE_STACK - 1) { ierr |= PHX_CSG_ERR_TRANCHE; break; }
                    tp++; tslice[tp] = loopTree; ttmin[tp] = tminAdvanced;
                    break;
                }
            }
            nodeIdx = PHX_POSTORDER_NEXT(nodeIdx, elevation);
        }
        if (ierr) break;
    }
    if (sp != 0) ierr |= PHX_CSG_ERR_END_EMPTY;
    isect = make_float4(0.f, 0.f, 0.f, 0.f);
    if (sp == 0) isect = stk[0];
    if (ierr) err |= PHX_STATUS_CSG_STACK;
    return isect.w > 0.f;
}

// one prim: leaf at the root, a boolean tree, or a list.  CV selects the FP64 root polish at
// compile time so the default path keeps the reference's FP32 expression structure.
template <int CV>
PHX_D bool intersect_prim(float4& isect, const PhxCsgCtx& g, int root, float t_min, const float3& o, const float3& d, unsigned& err)
{
    const unsigned typecode = __float_as_uint(__ldg(g.node + 4 * root + 3).z);
    isect = make_float4(0.f, 0.f, 0.f, 0.f);
    if (typecode >= PHX_CSG_LEAF) return intersect_leaf<CV>(isect, g, root, t_min, o, d, err);
    if (typecode < PHX_CSG_NODE) return intersect_tree<CV>(isect, g, root, t_min, o, d, err);
    if constexpr (PHX_CV_F(CV)) return intersect_list<CV>(isect, g, root, root, typecode, t_min, o, d, err);
    return false;
}
