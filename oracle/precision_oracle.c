/*
 * precision_oracle.c -- FP64 references of the precision mode (test
 * infrastructure only: the checker of the CUDA path's flagged FP64 narrow
 * phase, contact points and distances).
 *
 *  - orc_tritri_sat64: the 17-axis separating-axis test of the FP32
 *    predicate (gProximity triangleIntersection2,
 *    Source/Externals/inc/gProximity/cuda_intersect_tritri.h:349-433, restated
 *    in bvhcd_oracle.c), evaluated in double with one rounding per operation
 *    (no contraction: built with -ffp-contract=off), the same operations in
 *    the same order as the CUDA kernel, so the two agree bit for bit.
 *  - orc_contact64: the intersection segment of two intersecting triangles,
 *    after Moeller, "A fast triangle-triangle intersection test", Journal of
 *    Graphics Tools 2(2), 1997: each triangle is cut by the other's plane, the
 *    two cuts are intervals on the planes' common line, and their overlap is
 *    the segment.  The contact point is its midpoint.
 *  - orc_tri_distance64: the distance between two disjoint triangles, the
 *    smallest of the six vertex-triangle and nine edge-edge distances
 *    (closest point on a triangle and closest points of two segments after
 *    Ericson, Real-Time Collision Detection, 2005, sections 5.1.5 and 5.1.9).
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "bvhcd_oracle.h"

typedef struct { double x, y, z; } d3;

static inline d3 dsub(d3 a, d3 b) { d3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static inline d3 dadd(d3 a, d3 b) { d3 r = {a.x + b.x, a.y + b.y, a.z + b.z}; return r; }
static inline d3 dscale(d3 a, double s) { d3 r = {a.x * s, a.y * s, a.z * s}; return r; }
static inline double ddot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline d3 dcross(d3 a, d3 b) {
    d3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    return r;
}
static inline d3 dload(const float *p) { d3 r = {p[0], p[1], p[2]}; return r; }

static inline int axis_overlap64(d3 ax, d3 p1, d3 p2, d3 p3, d3 q1, d3 q2, d3 q3) {
    double P1 = ddot(ax, p1), P2 = ddot(ax, p2), P3 = ddot(ax, p3);
    double Q1 = ddot(ax, q1), Q2 = ddot(ax, q2), Q3 = ddot(ax, q3);
    double mx1 = fmax(fmax(P1, P2), P3), mn1 = fmin(fmin(P1, P2), P3);
    double mx2 = fmax(fmax(Q1, Q2), Q3), mn2 = fmin(fmin(Q1, Q2), Q3);
    return !(mn1 > mx2) && !(mn2 > mx1);
}

int orc_tritri_sat64(const float *P, const float *Q) {
    d3 P1 = dload(P), P2 = dload(P + 3), P3 = dload(P + 6);
    d3 Q1 = dload(Q), Q2 = dload(Q + 3), Q3 = dload(Q + 6);
    d3 p1 = {0.0, 0.0, 0.0};
    d3 p2 = dsub(P2, P1), p3 = dsub(P3, P1);
    d3 q1 = dsub(Q1, P1), q2 = dsub(Q2, P1), q3 = dsub(Q3, P1);
    d3 e[3] = {dsub(p2, p1), dsub(p3, p2), dsub(p1, p3)};
    d3 f[3] = {dsub(q2, q1), dsub(q3, q2), dsub(q1, q3)};
    d3 n = dcross(e[0], e[1]), m = dcross(f[0], f[1]);
    if (!axis_overlap64(n, p1, p2, p3, q1, q2, q3)) return 0;
    if (!axis_overlap64(m, p1, p2, p3, q1, q2, q3)) return 0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            if (!axis_overlap64(dcross(e[i], f[j]), p1, p2, p3, q1, q2, q3)) return 0;
    for (int i = 0; i < 3; i++)
        if (!axis_overlap64(dcross(e[i], n), p1, p2, p3, q1, q2, q3)) return 0;
    for (int j = 0; j < 3; j++)
        if (!axis_overlap64(dcross(f[j], m), p1, p2, p3, q1, q2, q3)) return 0;
    return 1;
}

/* points of triangle t on the plane (n, d): vertices on it, edge crossings */
static int cut_by_plane(const d3 t[3], const double dist[3], d3 out[3]) {
    int k = 0;
    for (int i = 0; i < 3; i++)
        if (dist[i] == 0.0 && k < 3) out[k++] = t[i];
    for (int i = 0; i < 3; i++) {
        int j = (i + 1) % 3;
        if ((dist[i] < 0.0 && dist[j] > 0.0) || (dist[i] > 0.0 && dist[j] < 0.0)) {
            double s = dist[i] / (dist[i] - dist[j]);
            if (k < 3) out[k++] = dadd(t[i], dscale(dsub(t[j], t[i]), s));
        }
    }
    return k;
}

int orc_contact64(const float *P, const float *Q, double *out4) {
    d3 p[3] = {dload(P), dload(P + 3), dload(P + 6)};
    d3 q[3] = {dload(Q), dload(Q + 3), dload(Q + 6)};
    d3 nP = dcross(dsub(p[1], p[0]), dsub(p[2], p[0]));
    d3 nQ = dcross(dsub(q[1], q[0]), dsub(q[2], q[0]));
    double dp[3], dq[3];
    for (int i = 0; i < 3; i++) {
        dp[i] = ddot(nQ, dsub(p[i], q[0]));
        dq[i] = ddot(nP, dsub(q[i], p[0]));
    }
    if ((dp[0] > 0 && dp[1] > 0 && dp[2] > 0) || (dp[0] < 0 && dp[1] < 0 && dp[2] < 0)) return 0;
    if ((dq[0] > 0 && dq[1] > 0 && dq[2] > 0) || (dq[0] < 0 && dq[1] < 0 && dq[2] < 0)) return 0;
    d3 D = dcross(nP, nQ);
    if (ddot(D, D) == 0.0) return 2; /* coplanar (or degenerate) */
    d3 a[3], b[3];
    int na = cut_by_plane(p, dp, a), nb = cut_by_plane(q, dq, b);
    if (na < 1 || nb < 1) return 0;
    if (na > 2) na = 2;
    if (nb > 2) nb = 2;
    if (na == 1) a[1] = a[0];
    if (nb == 1) b[1] = b[0];
    double ta0 = ddot(D, a[0]), ta1 = ddot(D, a[1]), tb0 = ddot(D, b[0]), tb1 = ddot(D, b[1]);
    if (ta0 > ta1) { d3 t = a[0]; a[0] = a[1]; a[1] = t; double s = ta0; ta0 = ta1; ta1 = s; }
    if (tb0 > tb1) { d3 t = b[0]; b[0] = b[1]; b[1] = t; double s = tb0; tb0 = tb1; tb1 = s; }
    d3 lo = ta0 >= tb0 ? a[0] : b[0];
    d3 hi = ta1 <= tb1 ? a[1] : b[1];
    double tlo = ta0 >= tb0 ? ta0 : tb0, thi = ta1 <= tb1 ? ta1 : tb1;
    if (tlo > thi) return 0;
    d3 c = dscale(dadd(lo, hi), 0.5);
    d3 d = dsub(hi, lo);
    out4[0] = c.x; out4[1] = c.y; out4[2] = c.z; out4[3] = sqrt(ddot(d, d));
    return 1;
}

/* closest point of triangle (a, b, c) to p, by Voronoi region */
static d3 closest_on_tri(d3 p, d3 a, d3 b, d3 c) {
    d3 ab = dsub(b, a), ac = dsub(c, a), ap = dsub(p, a);
    double d1 = ddot(ab, ap), d2 = ddot(ac, ap);
    if (d1 <= 0.0 && d2 <= 0.0) return a;
    d3 bp = dsub(p, b);
    double d3_ = ddot(ab, bp), d4 = ddot(ac, bp);
    if (d3_ >= 0.0 && d4 <= d3_) return b;
    double vc = d1 * d4 - d3_ * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3_ <= 0.0) return dadd(a, dscale(ab, d1 / (d1 - d3_)));
    d3 cp = dsub(p, c);
    double d5 = ddot(ab, cp), d6 = ddot(ac, cp);
    if (d6 >= 0.0 && d5 <= d6) return c;
    double vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) return dadd(a, dscale(ac, d2 / (d2 - d6)));
    double va = d3_ * d6 - d5 * d4;
    if (va <= 0.0 && (d4 - d3_) >= 0.0 && (d5 - d6) >= 0.0)
        return dadd(b, dscale(dsub(c, b), (d4 - d3_) / ((d4 - d3_) + (d5 - d6))));
    double den = 1.0 / (va + vb + vc);
    double v = vb * den, w = vc * den;
    return dadd(a, dadd(dscale(ab, v), dscale(ac, w)));
}

static double clamp01(double x) { return x < 0.0 ? 0.0 : (x > 1.0 ? 1.0 : x); }

/* squared distance between segments (p1, q1) and (p2, q2) */
static double seg_seg2(d3 p1, d3 q1, d3 p2, d3 q2) {
    d3 d1 = dsub(q1, p1), d2 = dsub(q2, p2), r = dsub(p1, p2);
    double a = ddot(d1, d1), e = ddot(d2, d2), f = ddot(d2, r);
    double s, t;
    if (a <= DBL_MIN && e <= DBL_MIN) return ddot(r, r);
    if (a <= DBL_MIN) {
        s = 0.0;
        t = clamp01(f / e);
    } else {
        double c = ddot(d1, r);
        if (e <= DBL_MIN) {
            t = 0.0;
            s = clamp01(-c / a);
        } else {
            double b = ddot(d1, d2), den = a * e - b * b;
            s = den != 0.0 ? clamp01((b * f - c * e) / den) : 0.0;
            t = (b * s + f) / e;
            if (t < 0.0) {
                t = 0.0;
                s = clamp01(-c / a);
            } else if (t > 1.0) {
                t = 1.0;
                s = clamp01((b - c) / a);
            }
        }
    }
    d3 c1 = dadd(p1, dscale(d1, s)), c2 = dadd(p2, dscale(d2, t));
    d3 d = dsub(c1, c2);
    return ddot(d, d);
}

double orc_tri_distance64(const float *P, const float *Q) {
    d3 p[3] = {dload(P), dload(P + 3), dload(P + 6)};
    d3 q[3] = {dload(Q), dload(Q + 3), dload(Q + 6)};
    double best = DBL_MAX;
    for (int i = 0; i < 3; i++) {
        d3 c = closest_on_tri(p[i], q[0], q[1], q[2]);
        d3 d = dsub(c, p[i]);
        double v = ddot(d, d);
        if (v < best) best = v;
        c = closest_on_tri(q[i], p[0], p[1], p[2]);
        d = dsub(c, q[i]);
        v = ddot(d, d);
        if (v < best) best = v;
    }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double v = seg_seg2(p[i], p[(i + 1) % 3], q[j], q[(j + 1) % 3]);
            if (v < best) best = v;
        }
    return sqrt(best);
}

static void tri9(const int *faces, const float *verts, int t, float *o9) {
    for (int k = 0; k < 3; k++) memcpy(o9 + 3 * k, verts + 3 * (size_t)faces[3 * (size_t)t + k], 12);
}

void orc_precision_pairs(int64_t n, const int *pairs, const int *faces, const float *verts, unsigned char *hit64,
                         double *contact4, double *dist) {
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < n; q++) {
        float a[9], b[9];
        tri9(faces, verts, pairs[2 * q], a);
        tri9(faces, verts, pairs[2 * q + 1], b);
        int h = orc_tritri_sat64(a, b);
        if (hit64) hit64[q] = (unsigned char)h;
        if (contact4) {
            double c[4] = {NAN, NAN, NAN, NAN};
            if (h) {
                int st = orc_contact64(a, b, c);
                if (st != 1) c[0] = c[1] = c[2] = c[3] = NAN;
            }
            memcpy(contact4 + 4 * q, c, sizeof(c));
        }
        if (dist) dist[q] = h ? 0.0 : orc_tri_distance64(a, b);
    }
}
