// proximity.cuh -- vertex-face and edge-edge proximities of a triangle pair.
//
// The reference carries the two measures a cloth solver builds its
// proximity constraints from, signed_vf_distance and signed_ee_distance
// (Mine/utility/CudaDeviceUtils.cu:163-193, with proj = v . (p0 x p1),
// Mine/utility/CudaDeviceUtils.h:66-68), but never calls them.  Here they are
// evaluated in FP64 with one rounding per operation (the operations and order
// of the CPU restatement in the oracle, so the two agree bit for bit) for the
// 15 feature pairs of a triangle pair: each vertex of either triangle against
// the other's face, and each edge of the first against each edge of the
// second.  A feature pair is a proximity when its signed distance is within
// the thickness and its closest points lie inside both features (every
// barycentric weight non-negative); feature pairs of one mesh that share a
// vertex id are skipped.
#pragma once

#include <cfloat>

#include "tritri.cuh"

namespace bvhcd {
namespace prox {

using prec::cross;
using prec::d3;
using prec::dot;
using prec::mk;
using prec::scale;
using prec::sub;

__device__ __forceinline__ d3 normalize(d3 v) { return scale(v, __ddiv_rn(1.0, __dsqrt_rn(dot(v, v)))); }
__device__ __forceinline__ double proj(d3 v, d3 p0, d3 p1) { return dot(v, cross(p0, p1)); }

// signed_vf_distance (x against the plane of y0, y1, y2) and
// signed_ee_distance (the lines of x0 x1 and y0 y1), split so that the parts
// shared by the feature pairs of one triangle pair are computed once (a
// face's normal, an edge's unit direction) and the signed distance is tested
// against the thickness before the weights are formed.  Every value is the
// same operations on the same operands as in the reference's formulas, so
// the results do not change.

// a face's unit normal; false for a degenerate face (the reference returns
// DBL_MAX)
__device__ __forceinline__ bool face_normal(d3 y0, d3 y1, d3 y2, d3 &n) {
    n = cross(normalize(sub(y1, y0)), normalize(sub(y2, y0)));
    if (!(dot(n, n) >= DBL_EPSILON)) return false;
    n = normalize(n);
    return true;
}
__device__ __forceinline__ void vf_weights(d3 x, d3 y0, d3 y1, d3 y2, d3 n, double w[4]) {
    const double b0 = proj(sub(y1, x), sub(y2, x), n);
    const double b1 = proj(sub(y2, x), sub(y0, x), n);
    const double b2 = proj(sub(y0, x), sub(y1, x), n);
    const double s = __dadd_rn(__dadd_rn(b0, b1), b2);
    w[0] = 1.0;
    w[1] = -__ddiv_rn(b0, s);
    w[2] = -__ddiv_rn(b1, s);
    w[3] = -__ddiv_rn(b2, s);
}
// the normal of two edges from their unit directions; false for parallel
// edges (the reference returns FLT_MAX below FLT_EPSILON)
__device__ __forceinline__ bool edge_normal(d3 ua, d3 ub, d3 &n) {
    n = cross(ua, ub);
    if (!(dot(n, n) >= (double)FLT_EPSILON)) return false;
    n = normalize(n);
    return true;
}
__device__ __forceinline__ void ee_weights(d3 x0, d3 x1, d3 y0, d3 y1, d3 n, double w[4]) {
    const double a0 = proj(sub(y1, x1), sub(y0, x1), n);
    const double a1 = proj(sub(y0, x0), sub(y1, x0), n);
    const double b0 = proj(sub(x0, y1), sub(x1, y1), n);
    const double b1 = proj(sub(x1, y0), sub(x0, y0), n);
    const double sa = __dadd_rn(a0, a1), sb = __dadd_rn(b0, b1);
    w[0] = __ddiv_rn(a0, sa);
    w[1] = __ddiv_rn(a1, sa);
    w[2] = -__ddiv_rn(b0, sb);
    w[3] = -__ddiv_rn(b1, sb);
}

struct Hit {
    int kind, fa, fb;
    double d;
    d3 n;
    double w[4];
};

// Calls emit(hit) for every proximity of triangles (ia, pa) and (ib, pb) in
// the order: kind 0 (vertex i of the first against the second's face, i =
// 0..2), kind 1 (vertex j of the second against the first's face), kind 2
// (edge i of the first, vertices i and i + 1 mod 3, against edge j of the
// second, i-major).  Vertex ids are compared only for two triangles of one
// mesh (same_mesh).
template <class Emit>
__device__ inline void triangle_pair(const int ia[3], const d3 pa[3], const int ib[3], const d3 pb[3],
                                     bool same_mesh, double h, Emit &&emit) {
    Hit r;
    d3 na, nb;
    const bool fa_ok = face_normal(pa[0], pa[1], pa[2], na);
    const bool fb_ok = face_normal(pb[0], pb[1], pb[2], nb);
    if (fb_ok)
        for (int i = 0; i < 3; i++) {
            if (same_mesh && (ia[i] == ib[0] || ia[i] == ib[1] || ia[i] == ib[2])) continue;
            r.d = dot(sub(pa[i], pb[0]), nb);
            if (!(fabs(r.d) <= h)) continue;
            vf_weights(pa[i], pb[0], pb[1], pb[2], nb, r.w);
            if (-r.w[1] >= 0.0 && -r.w[2] >= 0.0 && -r.w[3] >= 0.0) {
                r.n = nb; r.kind = 0; r.fa = i; r.fb = -1;
                emit(r);
            }
        }
    if (fa_ok)
        for (int j = 0; j < 3; j++) {
            if (same_mesh && (ib[j] == ia[0] || ib[j] == ia[1] || ib[j] == ia[2])) continue;
            r.d = dot(sub(pb[j], pa[0]), na);
            if (!(fabs(r.d) <= h)) continue;
            vf_weights(pb[j], pa[0], pa[1], pa[2], na, r.w);
            if (-r.w[1] >= 0.0 && -r.w[2] >= 0.0 && -r.w[3] >= 0.0) {
                r.n = na; r.kind = 1; r.fa = -1; r.fb = j;
                emit(r);
            }
        }
    d3 ua[3], ub[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        ua[k] = normalize(sub(pa[k == 2 ? 0 : k + 1], pa[k]));
        ub[k] = normalize(sub(pb[k == 2 ? 0 : k + 1], pb[k]));
    }
    for (int i = 0; i < 3; i++) {
        const int i1 = i == 2 ? 0 : i + 1;
        for (int j = 0; j < 3; j++) {
            const int j1 = j == 2 ? 0 : j + 1;
            if (same_mesh && (ia[i] == ib[j] || ia[i] == ib[j1] || ia[i1] == ib[j] || ia[i1] == ib[j1])) continue;
            if (!edge_normal(ua[i], ub[j], r.n)) continue;
            r.d = dot(sub(pa[i], pb[j]), r.n);
            if (!(fabs(r.d) <= h)) continue;
            ee_weights(pa[i], pa[i1], pb[j], pb[j1], r.n, r.w);
            if (r.w[0] >= 0.0 && r.w[1] >= 0.0 && -r.w[2] >= 0.0 && -r.w[3] >= 0.0) {
                r.kind = 2; r.fa = i; r.fb = j;
                emit(r);
            }
        }
    }
}

}  // namespace prox
}  // namespace bvhcd
