// tritri.cuh -- triangle-pair predicates and measures of the precision mode.
//
// * tritri_sat32_certain: the FP32 17-axis separating-axis test of the
//   narrow phase (the axes and overlap rule of gProximity's
//   triangleIntersection2, Source/Externals/inc/gProximity/
//   cuda_intersect_tritri.h:349-433), returning its answer only when it is
//   certain: every axis's separation margin g = max(min1 - max2, min2 - max1)
//   is compared with a bound on its rounding error, tau = 256 u B R (u =
//   2^-24; R the largest 1-norm of the six vertices after the translation to
//   the first one; B = |a|_1 |b|_1 for an axis a x b, |e|_1 |e0|_1 |e1|_1 for
//   the axes built on a face normal).  An axis with g > tau separates for
//   certain (no hit); if every axis has g < -tau the triangles overlap for
//   certain; otherwise the pair is flagged.
// * tritri_sat64: the same test in FP64, one rounding per operation, the
//   operations and order of the CPU reference, so the two agree bit for bit.
// * contact_point: midpoint and length of the intersection segment of two
//   intersecting triangles (each triangle cut by the other's plane; the two
//   cuts overlap on the planes' common line -- Moeller, "A fast
//   triangle-triangle intersection test", JGT 2(2), 1997), in FP32 or FP64.
// * tri_distance: distance of two disjoint triangles, the smallest of the six
//   vertex-triangle and nine edge-edge distances (closest points after
//   Ericson, Real-Time Collision Detection, 2005, 5.1.5 and 5.1.9).
#pragma once

#include <cfloat>

namespace bvhcd {
namespace prec {

// ------------------------------------------------------------ FP64, no contraction
struct d3 {
    double x, y, z;
};
__device__ __forceinline__ d3 mk(double x, double y, double z) { return d3{x, y, z}; }
__device__ __forceinline__ d3 sub(d3 a, d3 b) { return mk(__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y), __dsub_rn(a.z, b.z)); }
__device__ __forceinline__ d3 add(d3 a, d3 b) { return mk(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y), __dadd_rn(a.z, b.z)); }
__device__ __forceinline__ d3 scale(d3 a, double s) { return mk(__dmul_rn(a.x, s), __dmul_rn(a.y, s), __dmul_rn(a.z, s)); }
__device__ __forceinline__ double dot(d3 a, d3 b) {
    return __dadd_rn(__dadd_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)), __dmul_rn(a.z, b.z));
}
__device__ __forceinline__ d3 cross(d3 a, d3 b) {
    return mk(__dsub_rn(__dmul_rn(a.y, b.z), __dmul_rn(a.z, b.y)), __dsub_rn(__dmul_rn(a.z, b.x), __dmul_rn(a.x, b.z)),
              __dsub_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}

__device__ __forceinline__ bool overlap64(d3 ax, d3 p1, d3 p2, d3 p3, d3 q1, d3 q2, d3 q3) {
    const double P1 = dot(ax, p1), P2 = dot(ax, p2), P3 = dot(ax, p3);
    const double Q1 = dot(ax, q1), Q2 = dot(ax, q2), Q3 = dot(ax, q3);
    const double mx1 = fmax(fmax(P1, P2), P3), mn1 = fmin(fmin(P1, P2), P3);
    const double mx2 = fmax(fmax(Q1, Q2), Q3), mn2 = fmin(fmin(Q1, Q2), Q3);
    return !(mn1 > mx2) && !(mn2 > mx1);
}

__device__ inline bool tritri_sat64(d3 P1, d3 P2, d3 P3, d3 Q1, d3 Q2, d3 Q3) {
    const d3 p1 = mk(0.0, 0.0, 0.0);
    const d3 p2 = sub(P2, P1), p3 = sub(P3, P1);
    const d3 q1 = sub(Q1, P1), q2 = sub(Q2, P1), q3 = sub(Q3, P1);
    const d3 e[3] = {sub(p2, p1), sub(p3, p2), sub(p1, p3)};
    const d3 f[3] = {sub(q2, q1), sub(q3, q2), sub(q1, q3)};
    const d3 n = cross(e[0], e[1]), m = cross(f[0], f[1]);
    if (!overlap64(n, p1, p2, p3, q1, q2, q3)) return false;
    if (!overlap64(m, p1, p2, p3, q1, q2, q3)) return false;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            if (!overlap64(cross(e[i], f[j]), p1, p2, p3, q1, q2, q3)) return false;
    for (int i = 0; i < 3; i++)
        if (!overlap64(cross(e[i], n), p1, p2, p3, q1, q2, q3)) return false;
    for (int j = 0; j < 3; j++)
        if (!overlap64(cross(f[j], m), p1, p2, p3, q1, q2, q3)) return false;
    return true;
}

// ------------------------------------------------------------ FP32 with certainty
struct f3 {
    float x, y, z;
};
__device__ __forceinline__ f3 fk(float x, float y, float z) { return f3{x, y, z}; }
__device__ __forceinline__ f3 sub(f3 a, f3 b) { return fk(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)); }
__device__ __forceinline__ float dot(f3 a, f3 b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ f3 cross(f3 a, f3 b) {
    return fk(__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)), __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
              __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}
__device__ __forceinline__ float norm1(f3 a) { return fabsf(a.x) + fabsf(a.y) + fabsf(a.z); }

// 0: separated for certain, 1: overlapping for certain, 2: undecided
__device__ __forceinline__ int axis_certain(f3 ax, float tau, f3 p2, f3 p3, f3 q1, f3 q2, f3 q3) {
    const float P2 = dot(ax, p2), P3 = dot(ax, p3);
    const float Q1 = dot(ax, q1), Q2 = dot(ax, q2), Q3 = dot(ax, q3);
    const float mx1 = fmaxf(fmaxf(0.f, P2), P3), mn1 = fminf(fminf(0.f, P2), P3);
    const float mx2 = fmaxf(fmaxf(Q1, Q2), Q3), mn2 = fminf(fminf(Q1, Q2), Q3);
    const float g = fmaxf(mn1 - mx2, mn2 - mx1);
    if (g > tau) return 0;
    if (g < -tau) return 1;
    return 2;
}

// 1 hit, 0 no hit (both certain), -1 flagged
__device__ inline int tritri_sat32_certain(f3 P1, f3 P2, f3 P3, f3 Q1, f3 Q2, f3 Q3) {
    const f3 z = fk(0.f, 0.f, 0.f);
    const f3 p2 = sub(P2, P1), p3 = sub(P3, P1);
    const f3 q1 = sub(Q1, P1), q2 = sub(Q2, P1), q3 = sub(Q3, P1);
    const f3 e[3] = {sub(p2, z), sub(p3, p2), sub(z, p3)};
    const f3 f[3] = {sub(q2, q1), sub(q3, q2), sub(q1, q3)};
    const float R = fmaxf(fmaxf(fmaxf(norm1(p2), norm1(p3)), fmaxf(norm1(q1), norm1(q2))), norm1(q3));
    const float u = 256.f * 5.9604645e-08f * R;
    const float ne[3] = {norm1(e[0]), norm1(e[1]), norm1(e[2])};
    const float nf[3] = {norm1(f[0]), norm1(f[1]), norm1(f[2])};
    const float bn = ne[0] * ne[1], bm = nf[0] * nf[1];
    const f3 n = cross(e[0], e[1]), m = cross(f[0], f[1]);
    bool undecided = false;
    int r = axis_certain(n, u * bn, p2, p3, q1, q2, q3);
    if (r == 0) return 0;
    undecided |= r == 2;
    r = axis_certain(m, u * bm, p2, p3, q1, q2, q3);
    if (r == 0) return 0;
    undecided |= r == 2;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            r = axis_certain(cross(e[i], f[j]), u * ne[i] * nf[j], p2, p3, q1, q2, q3);
            if (r == 0) return 0;
            undecided |= r == 2;
        }
#pragma unroll
    for (int i = 0; i < 3; i++) {
        r = axis_certain(cross(e[i], n), u * ne[i] * bn, p2, p3, q1, q2, q3);
        if (r == 0) return 0;
        undecided |= r == 2;
    }
#pragma unroll
    for (int j = 0; j < 3; j++) {
        r = axis_certain(cross(f[j], m), u * nf[j] * bm, p2, p3, q1, q2, q3);
        if (r == 0) return 0;
        undecided |= r == 2;
    }
    return undecided ? -1 : 1;
}

// ------------------------------------------------------------ contact point / distance
// Generic over float / double through a tiny vector type.
template <typename F>
struct V {
    F x, y, z;
    __device__ V operator-(const V &b) const { return V{x - b.x, y - b.y, z - b.z}; }
    __device__ V operator+(const V &b) const { return V{x + b.x, y + b.y, z + b.z}; }
    __device__ V operator*(F s) const { return V{x * s, y * s, z * s}; }
};
template <typename F>
__device__ __forceinline__ F vdot(const V<F> &a, const V<F> &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename F>
__device__ __forceinline__ V<F> vcross(const V<F> &a, const V<F> &b) {
    return V<F>{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

template <typename F>
__device__ inline int cut_by_plane(const V<F> t[3], const F d[3], V<F> out[2]) {
    int k = 0;
    for (int i = 0; i < 3; i++)
        if (d[i] == F(0) && k < 2) out[k++] = t[i];
    for (int i = 0; i < 3; i++) {
        const int j = (i + 1) % 3;
        if (((d[i] < F(0) && d[j] > F(0)) || (d[i] > F(0) && d[j] < F(0))) && k < 2)
            out[k++] = t[i] + (t[j] - t[i]) * (d[i] / (d[i] - d[j]));
    }
    return k;
}

// 1: segment found (out = midpoint, length), 0: none, 2: coplanar;
// `cond` receives sin^2 of the angle between the planes (conditioning)
template <typename F>
__device__ inline int contact_point(const V<F> p[3], const V<F> q[3], F out[4], F *cond) {
    const V<F> nP = vcross(p[1] - p[0], p[2] - p[0]);
    const V<F> nQ = vcross(q[1] - q[0], q[2] - q[0]);
    F dp[3], dq[3];
    for (int i = 0; i < 3; i++) {
        dp[i] = vdot(nQ, p[i] - q[0]);
        dq[i] = vdot(nP, q[i] - p[0]);
    }
    if ((dp[0] > 0 && dp[1] > 0 && dp[2] > 0) || (dp[0] < 0 && dp[1] < 0 && dp[2] < 0)) return 0;
    if ((dq[0] > 0 && dq[1] > 0 && dq[2] > 0) || (dq[0] < 0 && dq[1] < 0 && dq[2] < 0)) return 0;
    const V<F> D = vcross(nP, nQ);
    const F dd = vdot(D, D), nn = vdot(nP, nP) * vdot(nQ, nQ);
    *cond = nn > F(0) ? dd / nn : F(0);
    if (dd == F(0)) return 2;
    V<F> a[2], b[2];
    int na = cut_by_plane(p, dp, a), nb = cut_by_plane(q, dq, b);
    if (na < 1 || nb < 1) return 0;
    if (na == 1) a[1] = a[0];
    if (nb == 1) b[1] = b[0];
    F ta0 = vdot(D, a[0]), ta1 = vdot(D, a[1]), tb0 = vdot(D, b[0]), tb1 = vdot(D, b[1]);
    if (ta0 > ta1) { const V<F> t = a[0]; a[0] = a[1]; a[1] = t; const F s = ta0; ta0 = ta1; ta1 = s; }
    if (tb0 > tb1) { const V<F> t = b[0]; b[0] = b[1]; b[1] = t; const F s = tb0; tb0 = tb1; tb1 = s; }
    const V<F> lo = ta0 >= tb0 ? a[0] : b[0];
    const V<F> hi = ta1 <= tb1 ? a[1] : b[1];
    const F tlo = ta0 >= tb0 ? ta0 : tb0, thi = ta1 <= tb1 ? ta1 : tb1;
    if (tlo > thi) return 0;
    const V<F> c = (lo + hi) * F(0.5), d = hi - lo;
    out[0] = c.x; out[1] = c.y; out[2] = c.z; out[3] = sqrt(vdot(d, d));
    return 1;
}

template <typename F>
__device__ inline V<F> closest_on_tri(V<F> p, V<F> a, V<F> b, V<F> c) {
    const V<F> ab = b - a, ac = c - a, ap = p - a;
    const F d1 = vdot(ab, ap), d2 = vdot(ac, ap);
    if (d1 <= F(0) && d2 <= F(0)) return a;
    const V<F> bp = p - b;
    const F d3 = vdot(ab, bp), d4 = vdot(ac, bp);
    if (d3 >= F(0) && d4 <= d3) return b;
    const F vc = d1 * d4 - d3 * d2;
    if (vc <= F(0) && d1 >= F(0) && d3 <= F(0)) return a + ab * (d1 / (d1 - d3));
    const V<F> cp = p - c;
    const F d5 = vdot(ab, cp), d6 = vdot(ac, cp);
    if (d6 >= F(0) && d5 <= d6) return c;
    const F vb = d5 * d2 - d1 * d6;
    if (vb <= F(0) && d2 >= F(0) && d6 <= F(0)) return a + ac * (d2 / (d2 - d6));
    const F va = d3 * d6 - d5 * d4;
    if (va <= F(0) && (d4 - d3) >= F(0) && (d5 - d6) >= F(0))
        return b + (c - b) * ((d4 - d3) / ((d4 - d3) + (d5 - d6)));
    const F den = F(1) / (va + vb + vc);
    return a + ab * (vb * den) + ac * (vc * den);
}

template <typename F>
__device__ __forceinline__ F clamp01(F x) { return x < F(0) ? F(0) : (x > F(1) ? F(1) : x); }

template <typename F>
__device__ inline F seg_seg2(V<F> p1, V<F> q1, V<F> p2, V<F> q2, F tiny) {
    const V<F> d1 = q1 - p1, d2 = q2 - p2, r = p1 - p2;
    const F a = vdot(d1, d1), e = vdot(d2, d2), f = vdot(d2, r);
    F s, t;
    if (a <= tiny && e <= tiny) return vdot(r, r);
    if (a <= tiny) {
        s = F(0);
        t = clamp01(f / e);
    } else {
        const F c = vdot(d1, r);
        if (e <= tiny) {
            t = F(0);
            s = clamp01(-c / a);
        } else {
            const F b = vdot(d1, d2), den = a * e - b * b;
            s = den != F(0) ? clamp01((b * f - c * e) / den) : F(0);
            t = (b * s + f) / e;
            if (t < F(0)) {
                t = F(0);
                s = clamp01(-c / a);
            } else if (t > F(1)) {
                t = F(1);
                s = clamp01((b - c) / a);
            }
        }
    }
    const V<F> d = (p1 + d1 * s) - (p2 + d2 * t);
    return vdot(d, d);
}

template <typename F>
__device__ inline F tri_distance(const V<F> p[3], const V<F> q[3], F tiny) {
    F best = F(3.0e38);
    for (int i = 0; i < 3; i++) {
        V<F> d = closest_on_tri(p[i], q[0], q[1], q[2]) - p[i];
        F v = vdot(d, d);
        best = v < best ? v : best;
        d = closest_on_tri(q[i], p[0], p[1], p[2]) - q[i];
        v = vdot(d, d);
        best = v < best ? v : best;
    }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            const F v = seg_seg2(p[i], p[(i + 1) % 3], q[j], q[(j + 1) % 3], tiny);
            best = v < best ? v : best;
        }
    return sqrt(best);
}

}  // namespace prec
}  // namespace bvhcd
